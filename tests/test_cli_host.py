"""Command-line program (programs/nutcracker, nutcracker.cpp:178-256): option
handling and input errors, no GPU (every case below stops before a chain is
created).  Exit statuses and messages follow the reference's main()."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "nutcracker-1_b200", "bin", "nutcracker_b200")
FIX = os.path.join(ROOT, "tests", "golden", "yaml")


def run(args, stdin=b"", cwd=None):
    if not os.path.exists(CLI):
        pytest.fail("command-line program not built: run nutcracker-1_b200/nutcracker_b200/build.py")
    return subprocess.run([CLI] + args, input=stdin, capture_output=True, cwd=cwd, timeout=60)


def test_help_listings_exit_1():
    r = run(["--help-modes"])
    assert r.returncode == 1 and b"'<v' - least value" in r.stderr and b"'>m' - largest magnitude" in r.stderr
    r = run(["--help-formats"])
    assert r.returncode == 1 and (b"The recognized input format types are:\n  - protobuf: Google Protocol Buffers "
                                  b"format\n  - yaml: YAML format") in r.stderr
    r = run(["--help"])
    assert r.returncode == 1 and b"--number-of-levels [ -n ]" in r.stderr and b"site-tolerance = 1e-10" in r.stderr


@pytest.mark.parametrize("args,message", [
    (["--optimizer-mode", "xx"], b"There is no such optimizer mode 'xx'."),
    (["--no-such-option"], b"unrecognised option '--no-such-option'"),
    (["-n"], b"the required argument for option '--number-of-levels' is missing"),
    (["--site-tolerance", "abc"], b"the argument ('abc') for option '--site-tolerance' is invalid"),
    # unsigned 32-bit options: values past the range fail as a conversion does
    (["-n", "4294967296"], b"the argument ('4294967296') for option '--number-of-levels' is invalid"),
    (["-n", "99999999999999999999"], b"the argument ('99999999999999999999') for option '--number-of-levels' is invalid"),
    (["-n", "-1"], b"the argument ('-1') for option '--number-of-levels' is invalid"),
])
def test_option_errors_exit_255(args, message):
    r = run(args)
    assert r.returncode == 255
    assert r.stderr.startswith(b"An error was encounted while parsing the options:") and message in r.stderr


@pytest.mark.parametrize("args,message", [
    (["--input-format", "hdf"], b"hdf is not a recognized/supported input format type."),
    (["--output-format", "text"], b"text is not a recognized/supported output format type."),
    (["--output-location", "a/b"], b"The output format type yaml does not support locations."),
    (["--input-format", "protobuf", "--input-location", "a"], b"The input format type protobuf does not support locations."),
    (["-f", "in.prb", "--input-location", "a"], b"The input format type protobuf does not support locations."),
    (["--output-states"], b"Output format yaml does not support outputing states."),
])
def test_format_errors_exit_255(args, message):
    with open(os.path.join(FIX, "external_field_5.yaml"), "rb") as f:
        r = run(args, stdin=f.read())
    assert r.returncode == 255 and message in r.stderr


def test_operator_errors_are_reported(tmp_path):
    bad = (b"sites:\n  - physical dimension: 2\n    left dimension: 1\n    right dimension: 1\n"
           b"    matrices:\n      - from: 1\n        to: 2\n        data: [1,0,0,1]\nsequence: [1]\n")
    r = run([], stdin=bad)
    assert r.returncode == 0 and b"The 'to' index is too high. (2 > 1)" in r.stderr and r.stdout == b""
    r = run(["--input-location", "nowhere"], stdin=open(os.path.join(FIX, "external_field_5.yaml"), "rb").read())
    assert b"No such location nowhere." in r.stderr
    r = run(["-f", str(tmp_path / "missing.yaml")])
    assert b"cannot open the input file" in r.stderr


def test_protobuf_input_errors(tmp_path):
    from nutcracker_b200 import capi
    b = capi.OperatorBuilder([2] * 3)
    b.add_term(capi.OperatorTerm.global_external_field(capi.Matrix.pauli("Z")))
    data = b.compile().serialize()
    r = run(["--input-format", "protobuf"], stdin=data[:-2])
    assert r.returncode == 0 and b"truncated" in r.stderr
    (tmp_path / "op.prb").write_bytes(data[:-2])
    r = run(["-f", str(tmp_path / "op.prb")])
    assert b"truncated" in r.stderr
    r = run(["--input-format", "protobuf"], stdin=b"")
    assert b"No operator sites were specified." in r.stderr


def test_configuration_file(tmp_path):
    (tmp_path / "nutcracker.cfg").write_text("# options\noptimizer-mode = zz\n")
    r = run([], cwd=tmp_path)
    assert r.returncode == 255 and b"There is no such optimizer mode 'zz'." in r.stderr
    # the command line wins over the configuration file
    r = run(["--optimizer-mode", "<v", "--input-format", "hdf"], cwd=tmp_path)
    assert r.returncode == 255 and b"hdf is not a recognized" in r.stderr
    (tmp_path / "other.cfg").write_text("bogus = 1\n")
    r = run(["-C", str(tmp_path / "other.cfg")], cwd=tmp_path)
    assert r.returncode == 255 and b"unrecognised option 'bogus' in the configuration file" in r.stderr


def test_option_forms():
    """--name=value and -nVALUE parse like the spaced forms; bad values are rejected."""
    r = run(["--optimizer-mode=zz"])
    assert r.returncode == 255 and b"There is no such optimizer mode 'zz'." in r.stderr
    r = run(["-nx"])
    assert r.returncode == 255 and b"the argument ('x') for option '--number-of-levels' is invalid" in r.stderr
    r = run(["--number-of-levels", "-3"])
    assert r.returncode == 255 and b"is invalid" in r.stderr
