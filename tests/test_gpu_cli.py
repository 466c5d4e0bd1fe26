"""Command-line program end to end on the GPU: the reference's README usage
(`generator | nutcracker -n 4`) on the transverse-Ising operator that the
reference's own generator emits (N=10, lambda=0.1), against the energies the
reference's tests pin (tests/chain.cpp:300-305, 418-430; tests/stress.cpp:107-186).
"""
import os
import subprocess

import pytest
import yaml

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "nutcracker-1_b200", "bin", "nutcracker_b200")
TFIM = os.path.join(ROOT, "tests", "golden", "yaml", "transverse_ising_0.1_10.yaml")
REF = [-10.022510957077, -8.213705725703, -8.188197237172, -8.148553771957]


def run(args, stdin=b"", cwd=None):
    return subprocess.run([CLI] + args, input=stdin, capture_output=True, cwd=cwd, timeout=600)


def test_piped_four_levels_match_reference_energies():
    # the options of the reference's four-level stress test (tests/stress.cpp:107-186:
    # initial bond dimension 2, site 1e-10, sweep and chain 1e-9, sanity 1e-12),
    # which pins these energies to 1e-7
    r = run(["-n", "4", "--initial-bandwidth", "2", "--site-tolerance", "1e-10", "--sweep-tolerance", "1e-9",
             "--chain-tolerance", "1e-9", "--sanity-tolerance", "1e-12", "--seed", "6"],
            stdin=open(TFIM, "rb").read())
    assert r.returncode == 0, r.stderr
    out = yaml.safe_load(r.stdout)
    conf = out["Configuration"]
    assert set(conf) == {"site convergence tolerance", "sweep convergence tolerance",
                         "chain convergence tolerance", "sanity check threshold"}
    levels = out["Energy levels"]
    assert len(levels) == 4, r.stderr
    for e, ref in zip(levels, REF):
        assert abs(e - ref) <= 1e-7 * abs(ref), (levels, REF)


@pytest.mark.parametrize("fixture,levels", [
    ("external_field_5.yaml", 4),           # README:25  external-field.py 5 | nutcracker -n 4
    ("transverse_ising_0.1_6.yaml", 3),     # README:32  transverse-ising-model.py 0.1 6 | nutcracker -n 3
    ("transverse_ising_0.1_10.yaml", 4),    # the ten-site chain of tests/stress.cpp, four levels
])
def test_readme_commands_at_default_options(fixture, levels):
    """No options at all: the reference's defaults (chain_options.cpp:21-30:
    initial bond dimension 1, every threshold 1e-12), sweeps until converged
    without a sweep bound as base_chain.cpp:112-123 does.  Energies against
    exact diagonalisation of the same YAML operator (1e-9 relative)."""
    from nutcracker_b200 import yaml_io
    from oracle import ed

    text = open(os.path.join(ROOT, "tests", "golden", "yaml", fixture), "rb").read()
    r = run(["-n", str(levels)], stdin=text)
    assert r.returncode == 0, r.stderr
    got = yaml.safe_load(r.stdout)["Energy levels"]
    assert len(got) == levels, r.stderr
    want, _ = ed.lowest_levels(yaml_io.read_operator(text), levels)
    for g, e in zip(got, want):
        assert abs(g - e) <= 1e-9 * max(abs(e), 1.0), (got, list(want))


def test_file_input_location_output_file_and_overwrite(tmp_path):
    nested = "problem:\n  hamiltonian:\n" + "".join(
        "    " + line + "\n" for line in open(TFIM).read().splitlines() if line and not line.startswith("---"))
    (tmp_path / "in.yaml").write_text(nested)
    (tmp_path / "nutcracker.cfg").write_text("chain-tolerance = 1e-10\n")
    out = tmp_path / "out.yaml"
    args = ["-f", str(tmp_path / "in.yaml"), "--input-location", "problem/hamiltonian", "-o", str(out)]
    r = run(args, cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    doc = yaml.safe_load(out.read_text())
    assert float(doc["Configuration"]["chain convergence tolerance"]) == 1e-10   # "1e-10" is a YAML string
    assert abs(doc["Energy levels"][0] - REF[0]) <= 1e-9 * abs(REF[0])
    r = run(args, cwd=tmp_path)   # exists, no --output-overwrite
    assert r.returncode == 0 and b"already exists." in r.stderr
    r = run(args + ["--output-overwrite", "--precision", "1"], cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    doc = yaml.safe_load(out.read_text())
    assert abs(doc["Energy levels"][0] - REF[0]) <= 1e-9 * abs(REF[0])


def test_protobuf_formats_end_to_end(tmp_path):
    """Operator in as an OperatorBuffer, results out as a SimulationResultsBuffer
    (nutcracker.proto) with an eigenvector state per level."""
    import struct

    from nutcracker_b200 import capi
    from test_capi_host import _fields

    b = capi.OperatorBuilder([2] * 10)
    b.add_term(capi.OperatorTerm.transverse_ising_field(capi.Matrix.pauli("Z"), 0.1 * capi.Matrix.pauli("X"),
                                                        capi.Matrix.pauli("X")))
    op = b.compile()
    (tmp_path / "op.prb").write_bytes(op.serialize())
    out = tmp_path / "res.prb"
    r = run(["-f", str(tmp_path / "op.prb"), "-o", str(out), "-n", "2"])
    assert r.returncode == 0, r.stderr
    fields = _fields(out.read_bytes())
    solutions = [v for f, w, v in fields if f == 1]
    thresholds = {f: struct.unpack("<d", v)[0] for f, w, v in fields if f in (2, 3, 4, 5)}
    assert len(solutions) == 2 and set(thresholds) == {2, 3, 4, 5}
    for k, sol in enumerate(solutions):
        sf = {f: v for f, w, v in _fields(sol)}
        e = struct.unpack("<d", sf[1])[0]
        assert abs(e - REF[k]) <= 1e-9 * abs(REF[k])
        state = capi.State.deserialize(sf[2])
        assert abs(state.overlap(state) - 1) < 1e-10
        assert abs(state.expectation(op) - e) < 1e-8 * abs(e)
