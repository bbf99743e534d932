"""Host-side input generators: splitmix64 known answers and the dam-break fields."""
import numpy as np

from vof_b200 import ic


def test_splitmix64_known_answers():
    # Published test vector of splitmix64 seeded with 0 (first three outputs).
    got = ic.splitmix64(0, 3)
    assert [int(x) for x in got] == [0xE220A8397B1DCDAF, 0x6E789E6AA1B965F4, 0x06C45D188009454F]


def test_uniform_range_and_determinism():
    a = ic.uniform(1, 10000, -1, 1)
    assert a.min() >= -1 and a.max() < 1
    assert np.array_equal(a, ic.uniform(1, 10000, -1, 1))
    assert abs(a.mean()) < 0.05


def test_normal_moments():
    z = ic.normal(3, 200000, std=2.0)
    assert abs(z.mean()) < 0.03 and abs(z.std() - 2.0) < 0.03


def test_dam_break_block_and_bc(V):
    prm = V.default_params(32, gy=0.0, gz=-9.81)
    F = ic.dam_break(prm)
    assert F.shape == (34, 34, 34) and F.dtype == np.float32
    inner = F[1:-1, 1:-1, 1:-1]
    # x, y: corner coordinate (i-1)*dx < 0.04 -> 13 cells; z: 19 full cells + 0.2
    assert np.all(inner[:19, :13, :13] == 1.0)
    assert np.allclose(inner[19, :13, :13], 0.2, atol=1e-6)
    assert np.all(inner[20:, :, :] == 0) and np.all(inner[:, 13:, :] == 0) and np.all(inner[:, :, 13:] == 0)
    assert np.array_equal(F[0], F[1]) and np.array_equal(F[:, :, 0], F[:, :, 1])


def test_dam_break_200_binary():
    class P:  # 200^3 geometry without loading the library
        nx = ny = nz = 200
        Lx = Ly = Lz = np.float32(0.1)

    F = ic.dam_break(P)
    assert set(np.unique(F)) <= {0.0, 1.0}
    assert F[1:-1, 1:-1, 1:-1].sum() == 80 * 80 * 120


def test_noisy_height_amplitude(V):
    prm = V.default_params(64)
    h = ic.noisy_height(prm, seed=1)
    assert h.shape == (66, 66)
    assert np.all(np.abs(h - 0.06) <= 0.5 * 0.1 / 64 + 1e-12)
    assert np.array_equal(h, ic.noisy_height(prm, seed=1))
    assert not np.array_equal(h, ic.noisy_height(prm, seed=2))


def test_sinusoidal_height(V):
    prm = V.default_params(40)
    h = ic.sinusoidal_height(prm, seed=5)
    assert np.isclose(np.abs(h - 0.06).max(), 0.1 / 40)


def test_random_state_properties(V):
    prm = V.default_params(10, 9, 8)
    s = ic.random_state(prm, seed=1)
    assert s["F"].min() == 0.0 and s["F"].max() == 1.0
    assert np.any(s["u"] == 0) and np.any(s["u"] > 0) and np.any(s["u"] < 0)
