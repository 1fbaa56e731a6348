"""Launch shapes change no result: every allowed value of every key of the
tuning table gives the mesh the defaults give (an adapt with fields, global
numbers and sliver layers, and its single-precision filtered twin)."""
import pytest

from conftest import build_gpu

pytestmark = pytest.mark.gpu


def test_every_tuning_value_gives_the_same_mesh():
    import omega_h_v1_b200 as G
    from omega_h_v1_b200 import tune
    L = tune._lib(G)
    defaults = tune.table(L)
    base = build_gpu(10, seed=4, pert=0.25, size=1 / 8., fields=True, parallel=True)

    def run(fp32):
        m = base.clone()
        m.set_fp32_filter(fp32)
        m.adapt(1 / 3., 0.3, 4, 50)
        d = m.digest()
        m.close()
        return d

    want = run(False), run(True)
    assert want[0] == want[1]
    try:
        for name, values in tune.CANDIDATES.items():
            for v in values:
                assert L.osh_b200_tuning_set(name.encode(), v) == 0
                assert (run(False), run(True)) == want, (name, v)
            assert L.osh_b200_tuning_set(name.encode(), defaults[name]) == 0
    finally:
        for k, v in defaults.items():
            L.osh_b200_tuning_set(k.encode(), v)
    base.close()
