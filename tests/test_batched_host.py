"""Host-side pieces of the batched form (no GPU): tile configurations, the
autotuner's table format and argument checks of nc_batch_create."""
import json

import numpy as np
import pytest

from oracle import mpo


def test_tile_configurations():
    from nutcracker_b200 import batched

    shapes = batched.tile_configs()
    assert len(shapes) >= 3
    assert all(r % 16 == 0 and c % 16 == 0 for r, c in shapes)


def test_committed_tile_table_is_valid():
    from nutcracker_b200 import batched

    entries = batched.load_tile_table()
    ncfg = len(batched.tile_configs())
    for stage, chi, D, d, cfg in entries:
        assert 0 <= stage < len(batched.STAGES)
        assert chi >= 1 and D >= 1 and d >= 1 and 0 <= cfg < ncfg


def test_tile_table_rejects_unknown_configuration(tmp_path):
    from nutcracker_b200 import batched

    p = tmp_path / "t.json"
    p.write_text(json.dumps({"entries": [{"stage": "heff_first", "chi": 16, "D": 5, "d": 2, "cfg": 99}]}))
    with pytest.raises(ValueError):
        batched.load_tile_table(str(p))
    p.write_text(json.dumps({"entries": [{"stage": "absorb", "chi": 64, "D": 5, "d": 2, "cfg": 1}]}))
    assert batched.load_tile_table(str(p)) == [(5, 64, 5, 2, 1)]


def test_batch_argument_checks_before_any_device_work():
    """Runs on a thread of its own: the library's error status is per host
    thread, and the failing calls here must not leave it set for later tests."""
    import threading

    from nutcracker_b200 import NutcrackerError
    from nutcracker_b200.batched import Batch

    ops = mpo.xxz_random(6, np.random.default_rng(0))
    seen = {}

    def body():
        for key, kw in (("krylov", {"krylov_dimension": 30}), ("precision", {"precision": 2})):
            try:
                Batch([ops], [4], **kw)
            except NutcrackerError as e:
                seen[key] = e.code
        try:
            Batch([ops], [4, 8])
        except ValueError:
            seen["count"] = True

    t = threading.Thread(target=body)
    t.start()
    t.join()
    assert seen == {"krylov": 1002, "precision": 1002, "count": True}
