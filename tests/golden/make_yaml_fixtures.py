"""Generate the YAML operator fixtures from the reference's own generator scripts.

Runs the reference's example generators (examples/generate/yaml/*.py, the
programs its README pipes into the `nutcracker` program) in this container and
stores their standard output under tests/golden/yaml/.  The fixtures exercise
the reference's input format as it is actually produced: document markers and
comments, anchors and aliases, real and [re, im] complex entries, repeated
sites through `sequence`.  Run from the repository root:

    python tests/golden/make_yaml_fixtures.py /path/to/reference
"""
import os
import subprocess
import sys

CASES = [  # (generator, arguments, fixture name)
    ("transverse-ising-model.py", ["0.1", "6"], "transverse_ising_0.1_6.yaml"),
    ("transverse-ising-model.py", ["0.1", "10"], "transverse_ising_0.1_10.yaml"),
    ("external-field.py", ["5"], "external_field_5.yaml"),
    ("external-field-using-anchors.py", ["5"], "external_field_anchors_5.yaml"),
    ("XY-ising-model.py", ["0.5", "7"], "xy_0.5_7.yaml"),
    ("Heisenberg-ising-model.py", ["1", "1", "8"], "heisenberg_1_1_8.yaml"),
    ("long-range-dipole-coupling-model.py", ["3", "6"], "dipole_3_6.yaml"),
]


def main(ref):
    here = os.path.dirname(os.path.abspath(__file__))
    out_dir = os.path.join(here, "yaml")
    os.makedirs(out_dir, exist_ok=True)
    for script, args, name in CASES:
        path = os.path.join(ref, "examples", "generate", "yaml", script)
        text = subprocess.run([sys.executable, path] + args, check=True, capture_output=True, text=True).stdout
        with open(os.path.join(out_dir, name), "w") as f:
            f.write(text)
        print(name, len(text), "bytes")


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("NUTCRACKER_REFERENCE", "")
    if not root:
        sys.exit("usage: make_yaml_fixtures.py <reference_root>  (or set NUTCRACKER_REFERENCE)")
    main(root)
