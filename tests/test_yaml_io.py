"""YAML operator format (yaml.cpp:169-306, io.hpp:350-370, README:27-187), no GPU.

The library's own reader is checked against the operators that the
reference's generator scripts emit (tests/golden/yaml/, made by
tests/golden/make_yaml_fixtures.py), parsed independently with PyYAML under
the reference's rules; the writer must round-trip; malformed operators must
fail with the reference's messages.  The transverse-Ising fixture at N=10,
lambda=0.1 must reproduce the energies that the reference's tests pin
(tests/chain.cpp:300-305, 418-430).
"""
import glob
import os

import numpy as np
import pytest
import yaml

from oracle import ed

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "yaml", "*.yaml")))


@pytest.fixture(scope="module")
def yio():
    from nutcracker_b200 import yaml_io
    return yaml_io


def _reference_semantics(text):
    """The operator under the reference's reading rules, parsed by PyYAML."""
    doc = yaml.safe_load(text)
    out = []
    for k in doc["sequence"]:
        u = doc["sites"][k - 1]
        links = []
        for m in u["matrices"]:
            data = [complex(x[0], x[1]) if isinstance(x, list) else
                    complex(x["real"], x["imag"]) if isinstance(x, dict) else complex(x) for x in m["data"]]
            links.append((m["from"], m["to"], data))
        out.append((u["physical dimension"], u["left dimension"], u["right dimension"], links))
    return out


@pytest.mark.parametrize("path", FIXTURES, ids=os.path.basename)
def test_reader_matches_reference_semantics(yio, path):
    text = open(path).read()
    sites = yio.read_operator(text)
    want = _reference_semantics(text)
    assert len(sites) == len(want)
    for s, (d, cl, cr, links) in zip(sites, want):
        assert (s.d, s.cl, s.cr, s.nnz) == (d, cl, cr, len(links))
        for n, (f, t, data) in enumerate(links):
            assert (s.idx[0, n], s.idx[1, n]) == (f, t)
            # the d*d list as written, into the column-major (d,d) block
            assert np.array_equal(s.W[:, :, n].ravel(order="F"), np.array(data))


@pytest.mark.parametrize("path", FIXTURES, ids=os.path.basename)
def test_writer_round_trip(yio, path):
    sites = yio.read_operator(open(path).read())
    text = yio.write_operator(sites)
    back = yio.read_operator(text)
    assert len(back) == len(sites)
    for a, b in zip(sites, back):
        assert (a.d, a.cl, a.cr) == (b.d, b.cl, b.cr)
        assert np.array_equal(a.idx, b.idx) and np.array_equal(a.W, b.W)
    # identical sites are listed once
    doc = yaml.safe_load(text)
    assert len(doc["sites"]) <= len(yaml.safe_load(open(path).read())["sites"])


def test_transverse_ising_fixture_gives_reference_energies(yio):
    sites = yio.read_operator(open(os.path.join(HERE, "golden", "yaml", "transverse_ising_0.1_10.yaml")).read())
    w, _ = ed.lowest_levels(sites, 4)
    ref = [-10.022510957077, -8.213705725703, -8.188197237172, -8.148553771957]
    assert np.allclose(w, ref, atol=1e-9)


def test_complex_entry_forms_and_location(yio):
    text = """
    --- # an operator nested in a larger document
    meta: {name: demo, tags: [a, b]}
    problem:
      hamiltonian:
        sequence: [1, 2]
        sites:
          - physical dimension: 2
            left dimension: 1
            right dimension: 2
            matrices:
              - {from: 1, to: 1, data: [1, 0, 0, 1]}
              - from: 1
                to: 2
                data: [0, [0, -1], {real: 0, imag: 1}, 0]   # Y
          - physical dimension: 2
            left dimension: 2
            right dimension: 1
            matrices:
              - from: 2
                to: 1
                data:
                  - 0
                  - [0, -1]
                  - [0, 1]
                  - 0
    """
    text = "\n".join(line[4:] for line in text.splitlines())
    sites = yio.read_operator(text, location="problem/hamiltonian")
    assert len(sites) == 2
    y = np.array([[0, -1j], [1j, 0]])
    assert np.array_equal(sites[0].W[:, :, 1], y.T)
    assert np.array_equal(sites[1].W[:, :, 0], y.T)
    assert sites[1].idx[:, 0].tolist() == [2, 1]
    from nutcracker_b200 import NutcrackerError
    with pytest.raises(NutcrackerError, match="No such location problem/missing."):
        yio.read_operator(text, location="problem/missing")


SITE_A = """  - physical dimension: 2
    left dimension: {cl}
    right dimension: {cr}
    matrices:
      - from: {f}
        to: {t}
        data: {data}
"""


def _doc(sites, sequence):
    return "sites:\n" + "".join(SITE_A.format(**s) for s in sites) + "sequence: %s\n" % sequence


def _site(cl=1, cr=1, f=1, t=1, data="[1,0,0,1]"):
    return dict(cl=cl, cr=cr, f=f, t=t, data=data)


@pytest.mark.parametrize("doc,message", [
    (_doc([_site(f=0)], "[1]"), "The 'from' index is too low. (0 < 1)"),
    (_doc([_site(f=2)], "[1]"), "The 'from' index is too high. (2 > 1)"),
    (_doc([_site(t=0)], "[1]"), "The 'to' index is too low. (0 < 1)"),
    (_doc([_site(cr=2, t=3)], "[1]"), "The 'to' index is too high. (3 > 2)"),
    (_doc([_site(data="[1,0,0]")], "[1]"), "The length of the data (3) does not match the correct length (4)."),
    (_doc([_site()], "[1, 3]"), "non-existent operator site number 2 appeared in the sequence."),
    (_doc([_site(cl=2, f=1)], "[1]"), "The left dimension of the left-most site must be one but instead is 2."),
    (_doc([_site(cr=2)], "[1]"), "The right dimension of the right-most site must be one but instead is 2."),
    (_doc([_site(cr=2), _site(cl=3, cr=1)], "[1, 2]"),
     "The left dimension (3) of site 0 does not match the right dimension (2) of site 1.  (3 != 2)"),
    (_doc([_site()], "[]"), "No operator sites were specified."),
    ("sites: []\n", "No operator sites were specified."),
])
def test_reference_error_messages(yio, doc, message):
    from nutcracker_b200 import NutcrackerError
    with pytest.raises(NutcrackerError) as e:
        yio.read_operator(doc)
    assert message in str(e.value)


def test_malformed_yaml_is_rejected(yio):
    from nutcracker_b200 import NutcrackerError
    for bad in ["sites:\n\t- physical dimension: 2\n", "sites: [1, 2\nsequence: [1]\n",
                "sites:\n  - physical dimension: 2\n    left dimension: 1\n    right dimension: 1\n"
                "    matrices:\n      - {from: 1, to: 1, data: *nope}\nsequence: [1]\n"]:
        with pytest.raises(NutcrackerError):
            yio.read_operator(bad)


def test_hostile_input_fails_with_a_message(yio):
    """Deep nesting is bounded (the parser recurses per level) and dimensions
    past the format's unsigned 32-bit range are rejected before any size
    computed from them is used."""
    from nutcracker_b200 import NutcrackerError
    for deep in ["[" * 100000, "- " * 100000 + "1", "a: " + "[" * 300 + "]" * 300 + "\n"]:
        with pytest.raises(NutcrackerError, match="nesting deeper than 256 levels"):
            yio.read_operator(deep)
    shallow = "sites: " + "[" * 200 + "]" * 200 + "\n"
    with pytest.raises(NutcrackerError, match="'sites' must be a list|every entry"):
        yio.read_operator(shallow)
    site = ("  - physical dimension: {d}\n    left dimension: 1\n    right dimension: 1\n    matrices:\n"
            "      - from: 1\n        to: 1\n        data: [1,0,0,1]\n")
    for d in (4294967296, 99999999999):
        with pytest.raises(NutcrackerError, match="below 2\\^32"):
            yio.read_operator("sequence: [1]\nsites:\n" + site.format(d=d))


def test_line_endings_quoted_keys_and_flow_documents(yio):
    text = open(os.path.join(HERE, "golden", "yaml", "external_field_anchors_5.yaml")).read()
    want = yio.read_operator(text)
    for variant in (text.replace("\n", "\r\n"), text.replace("physical dimension", '"physical dimension"')):
        got = yio.read_operator(variant)
        assert all(np.array_equal(a.W, b.W) and np.array_equal(a.idx, b.idx) for a, b in zip(got, want))
    flow = ("{sites: [{physical dimension: 2, left dimension: 1, right dimension: 1, "
            "matrices: [{from: 1, to: 1, data: [1, 0, 0, -1]}]}], sequence: [1]}")
    (s,) = yio.read_operator(flow)
    assert np.array_equal(s.W[:, :, 0], np.diag([1, -1]))


@pytest.mark.parametrize("name", ["heisenberg", "spin1", "xxz"])
def test_reader_reads_the_oracles_yaml(yio, name):
    """Operators written by the oracle's own YAML emitter read back identically."""
    from oracle import mpo
    ops = {"heisenberg": lambda: mpo.heisenberg(7), "spin1": lambda: mpo.heisenberg_spin1(5, 0.5),
           "xxz": lambda: mpo.xxz_random(6, np.random.default_rng(3))}[name]()
    got = yio.read_operator(mpo.to_yaml(ops))
    assert len(got) == len(ops)
    for a, b in zip(got, ops):
        assert (a.d, a.cl, a.cr) == (b.d, b.cl, b.cr)
        assert np.array_equal(a.idx, b.idx) and np.allclose(a.W, b.W, rtol=0, atol=0)
