"""The seeded uneven sweep's members (host logic of the batched engine):
deterministic, within the stated ranges, zones on the grid, boxes bucketed."""
import numpy as np

from multicellular_phase_field_active_gel_organoids_b200 import batched as B


def test_members_deterministic_and_in_range():
    a = B.sweep_members(64, seed=1)
    b = B.sweep_members(64, seed=1)
    assert [m.N for m in a] == [m.N for m in b]
    assert all(np.array_equal(x.centres, y.centres) for x, y in zip(a, b))
    for m in a:
        assert m.N in B.GRIDS
        assert 16.0 <= m.radius <= 32.0
        assert 1 <= m.ncells <= 128
        assert m.box % 16 == 0 and 64 <= m.box <= 128 and m.box >= 4 * m.radius
        assert 0.5 <= m.contract <= 2.0 and 0.5 <= m.turnover <= 2.0
        # every zone [xc - z, xc + z) and FFT box on the grid with a margin
        lo = m.centres.min(axis=0) - m.zone_size
        hi = m.centres.max(axis=0) + m.zone_size
        assert lo.min() >= 1 and hi.max() <= m.N - 1


def test_member_parameters():
    m = B.sweep_members(4, seed=1)[2]
    p = m.config().params()
    assert p["N_s"] == m.N and p["N_ini"] == m.ncells and p["zone_size"] == m.zone_size
    assert np.isclose(p["a_ort_apical"], 100.0 * m.contract)
    assert np.isclose(p["a_tan_apical"], p["a_ort_apical"] * p["epsilon_ap"])
    assert np.isclose(p["degrate_apical"], 100.0 * m.turnover)
    assert np.isclose(p["degrate_basal"], p["degrate_apical"])
    assert np.isclose(p["matgenrate_basal"], p["matgenrate_apical"])


def test_buckets_group_box_grid_and_size_class():
    ms = B.sweep_members(256, seed=1)
    keys = {m.bucket() for m in ms}
    assert {int(k.split("_")[0][1:]) for k in keys} <= {64, 80, 96, 112, 128}
    for m in ms:
        assert m.bucket().startswith(f"M{m.box}_N{m.N}_")
    assert B.box_for_radius(16.0) == 64 and B.box_for_radius(16.01) == 80 and B.box_for_radius(32.0) == 128
