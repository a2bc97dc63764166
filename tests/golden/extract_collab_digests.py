"""Writes collab_recorded.json: the NL4D group-filter digests the reference records in
av-denoise-core/src/collab/tests/fused/recorded.rs (covered pixels, mean, RMS, mean group
weight and eight probe pixels per case), keyed by the case label.

Usage: python extract_collab_digests.py <path to the reference's collab/tests/fused/recorded.rs>.
Run where a reference checkout is available; the JSON it writes is committed, and nothing reads the
reference at test time.
"""

import json
import re
import sys
from pathlib import Path

if len(sys.argv) != 2:
    sys.exit("usage: extract_collab_digests.py <reference av-denoise-core/src/collab/tests/fused/recorded.rs>")
SRC = Path(sys.argv[1])
OUT = Path(__file__).with_name("collab_recorded.json")

text = SRC.read_text()
cases = {}
for m in re.finditer(r"let want = Digest \{(.*?)\};(.*?)(?:\(\"([^\"]+)\", setup, want\)|"
                     r"assert_matches_recorded\(\"([^\"]+)\")", text, re.S):
    body, _, label, label2 = m.groups()
    label = label or label2
    covered = int(re.search(r"covered:\s*(\d+)", body).group(1))
    fields = {k: float(re.search(k + r":\s*([0-9.eE+-]+)", body).group(1))
              for k in ("pixel_mean", "pixel_rms", "weight_mean")}
    probes = [float(x) for x in re.findall(r"([0-9]+\.[0-9]+)", re.search(r"probes:\s*\[(.*?)\]", body, re.S).group(1))]
    cases[label] = {"covered": covered, **fields, "probes": probes}

OUT.write_text(json.dumps(cases, indent=1) + "\n")
print(f"wrote {len(cases)} cases to {OUT}")
