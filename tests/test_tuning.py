"""The tuning table of launch shapes (no GPU needed): names, defaults,
allowed values, and the table file's format and failure behaviour."""
import ctypes as C

import omega_h_v1_b200 as G
from omega_h_v1_b200 import tune


def _L():
    return tune._lib(G)


def test_every_key_has_its_stated_values():
    L = _L()
    names = [L.osh_b200_tuning_name(i).decode() for i in range(L.osh_b200_tuning_count())]
    assert names == list(tune.CANDIDATES) + list(tune.OTHER_KEYS)
    for name, values in list(tune.CANDIDATES.items()) + list(tune.OTHER_KEYS.items()):
        v = C.c_uint()
        assert L.osh_b200_tuning_get(name.encode(), C.byref(v)) == 0
        assert v.value in values


def test_set_rejects_unknown_names_and_values():
    L = _L()
    assert L.osh_b200_tuning_set(b"carry_group", 3) == 4
    assert L.osh_b200_tuning_set(b"no_such_key", 8) == 4
    v = C.c_uint()
    assert L.osh_b200_tuning_get(b"no_such_key", C.byref(v)) == 4


def test_table_file(tmp_path):
    L = _L()
    L.osh_b200_tuning_load.restype = C.c_int
    L.osh_b200_tuning_load.argtypes = [C.c_char_p]
    before = tune.table(L)
    good = tmp_path / "good.txt"
    good.write_text("# a comment\n\ncarry_group 16   # trailing comment\nscan_items 8\n")
    assert L.osh_b200_tuning_load(str(good).encode()) == 0
    t = tune.table(L)
    assert t["carry_group"] == 16 and t["scan_items"] == 8
    bad = tmp_path / "bad.txt"
    bad.write_text("carry_group 4\ngather_block 100\n")
    assert L.osh_b200_tuning_load(str(bad).encode()) == 4
    assert tune.table(L)["carry_group"] == 16          # nothing of a bad file applied
    assert L.osh_b200_tuning_load(str(tmp_path / "missing.txt").encode()) == 9
    for k, v in before.items():
        assert L.osh_b200_tuning_set(k.encode(), v) == 0
    assert tune.table(L) == before
