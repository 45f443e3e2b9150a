"""Host logic of the autotuner (openatom_b200.tuner): table keys, lookup,
candidate sets.  No GPU."""
import json

from openatom_b200 import tuner
from openatom_b200.system import make_system


def test_system_key_and_lookup(tmp_path):
    s = make_system("w8", seed=3)
    k = tuner.system_key(s, "mixed")
    assert k == f"mixed/64x64x64/s{s.nstate}/g{s.ng}/nl{len(s.nl_atoms())}"
    assert tuner.system_key(make_system("w8", seed=4), "mixed") == k   # positions do not enter
    path = tmp_path / "t.json"
    choice = {"group_pair": 3, "group_state": 4, "dgemm_kblocks": 96, "tgemm_kblocks": 32, "fft_path": 1}
    path.write_text(json.dumps({"meta": {}, "entries": {k: {"choice": choice}}}))
    assert tuner.lookup(s, "mixed", path=str(path)) == choice
    assert tuner.lookup(s, "fp64", path=str(path)) is None


def test_candidates_respect_sizes():
    s = make_system("w2", seed=3)
    caps = {"dgemm_kblocks": 160, "tgemm_kblocks": 64}
    cur = {}
    assert max(tuner.candidates("group_pair", s, "mixed", cur, caps)) <= (s.nstate + 1) // 2
    assert max(tuner.candidates("group_state", s, "fp64", cur, caps)) <= s.nstate
    assert all(2 <= k <= 160 for k in tuner.candidates("dgemm_kblocks", s, "fp64", cur, caps))
    assert all(1 <= k <= 64 for k in tuner.candidates("tgemm_kblocks", s, "mixed", cur, caps))
    assert tuner.candidates("fft_path", s, "mixed", cur, caps) == [1]
    assert tuner.candidates("fft_path", s, "fp64", cur, caps) == [1, 2]
    assert "fft_path" not in tuner.knobs_for("mixed")
    assert "tgemm_kblocks" not in tuner.knobs_for("mixed")


def test_committed_table_is_well_formed():
    tab = tuner.load_table()
    fields = {"group_state", "group_pair", "dgemm_kblocks", "tgemm_kblocks", "fft_path"}
    for key, e in tab.items():
        prec = key.split("/")[0]
        assert prec in ("mixed", "fp64")
        assert set(e["choice"]) == fields
        assert e["ms_tuned"] <= e["ms_default"] * 1.05
        if prec == "mixed":
            assert e["choice"]["fft_path"] == 1
