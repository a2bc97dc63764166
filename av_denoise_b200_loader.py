"""Imports the `av-denoise_b200/` package directory as the module `av_denoise_b200`.

The directory name carries a hyphen, which `import` cannot spell, so consumers call `load()`.
"""

from __future__ import annotations

import importlib.util
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent
PKG_DIR = ROOT / "av-denoise_b200"


def load():
    mod = sys.modules.get("av_denoise_b200")
    if mod is not None:
        return mod
    spec = importlib.util.spec_from_file_location(
        "av_denoise_b200", PKG_DIR / "__init__.py", submodule_search_locations=[str(PKG_DIR)]
    )
    mod = importlib.util.module_from_spec(spec)
    sys.modules["av_denoise_b200"] = mod
    spec.loader.exec_module(mod)
    return mod
