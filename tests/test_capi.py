"""CPU-only checks of the C ABI library: it loads without a GPU, exports every
entry point the headers declare (the reference's omega_h.h set included), and
its host-side helpers (box generator, swap tables) agree with the oracle's."""
import ctypes as C
import subprocess

import numpy as np
import pytest

from conftest import ROOT, cuda_available, radial_size_np

# every function of the reference's public header (include/omega_h.h:12-78)
REFERENCE_API = [
    "osh_init", "osh_fini", "osh_free", "osh_read_vtk", "osh_write_vtk", "osh_new",
    "osh_build_ents", "osh_dim", "osh_nelems", "osh_nverts", "osh_count", "osh_down",
    "osh_up", "osh_up_offs", "osh_up_dirs", "osh_star", "osh_star_offs", "osh_coords",
    "osh_own_rank", "osh_own_id", "osh_global", "osh_new_field", "osh_get_field",
    "osh_free_field", "osh_nfields", "osh_field", "osh_components", "osh_new_label",
    "osh_get_label", "osh_free_label", "osh_new_global", "osh_accumulate_to_owner",
    "osh_conform", "osh_mark_classified", "osh_ghost", "osh_num_ghost_layers",
    "osh_adapt", "osh_identity_size"]


def G():
    import omega_h_v1_b200
    return omega_h_v1_b200


def test_library_exports_every_declared_symbol():
    lib = G().LIB_PATH
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True,
                         text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    declared = G().exported_symbols()
    missing = [s for s in declared if s not in exported]
    assert not missing, missing
    assert set(REFERENCE_API) <= set(declared)
    # nothing else leaks out of the library
    extra = [s for s in exported if s.startswith("osh_") and s not in declared]
    assert not extra, extra


def test_library_loads_and_binds():
    L = G().lib()
    for s in G().exported_symbols():
        assert hasattr(L, s)


@pytest.mark.parametrize("n,seed,pert", [(1, 0, 0.1), (4, 3, 0.2), (9, 11, 0.3)])
def test_box_generator_matches_oracle(n, seed, pert):
    from oracle import oracle as O
    a = G().box(n, seed, pert)
    b = O.box(n, seed, pert)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_radial_size_matches_oracle():
    from oracle import oracle as O
    coords, _, center = O.box(6, 2, 0.1)
    assert np.array_equal(radial_size_np(coords, center, 0.01, 0.04),
                          O.radial_size(coords, center, 0.01, 0.04))


def test_swap_tables_match_oracle():
    from oracle import oracle as O
    for rs in range(3, 8):
        for x, y in zip(G().swap_table(rs), O.swap_table(rs)):
            assert np.array_equal(x, y)


@pytest.mark.skipif(cuda_available(), reason="checks the no-device error path")
def test_no_device_reports_error_instead_of_aborting():
    L = G().lib()
    h = L.osh_new(3)
    assert not h
    assert L.osh_b200_last_error() in (1, 5)
    L.osh_b200_clear_error()
    assert L.osh_b200_last_error() == 0
