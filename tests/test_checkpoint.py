"""Restart files: the reference's conf_new/conf_old text records
(store_config.f90:20-67, init_config.f90:104-209) and the exact binary
side-car."""
import numpy as np
import pytest

from mfa_b200 import _abi, checkpoint
from mfa_b200._abi import FP64
from oracle import Oracle


def test_conf_records_follow_the_fortran_formats(tmp_path):
    """Every record with the widths of the reference's formats: '(i1)',
    '(4i10)', 120 = (2i10), 110 = (i3), 113 = (i3,3f13.7), 103 = (3f15.7),
    130 = (3i13)."""
    path = tmp_path / "conf_new"
    r0 = np.array([[1.5, -0.25, 10.0], [58.4237, 1.23e-8, 59.99999996]])
    v = np.array([[0.5, -1.0, 2.25], [0.0, 0.0, -3.125]])
    a = np.array([[100.0, -0.0000001, 0.0], [1.0, 2.0, 3.0]])
    walls = {"r0_twall": [0.0, 0.0, 60.0], "rx_twall": np.array([[0.005, 0.0], [0.0, 0.0], [0.0, 0.0]]),
             "pbc_twall": [1, 0, -2], "s_force_grad": [0, 0, 1]}
    checkpoint.write_conf(str(path), r0, v, a, [1, 3], n_mon=2, n_chain=1, n_mon_d=1, n_chain_d=0,
                          n_cell_w=(4, 5), walls=walls, dt=0.005)
    lines = path.read_text().split("\n")
    assert lines[:4] == ["1", "         2         1         1         0", "         4         5", "  2"]
    assert lines[4] == "  1    1.5000000   -0.2500000   10.0000000"
    assert lines[5] == "  3   58.4237000    0.0000000   60.0000000"
    assert lines[6] == "      0.5000000     -1.0000000      2.2500000"
    assert lines[7] == "      0.0000000      0.0000000     -3.1250000"
    assert lines[8] == "    100.0000000     -0.0000001      0.0000000"
    assert lines[10] == "      0.0000000      0.0000000     60.0000000"       # r0_twall
    assert lines[11] == "      1.0000000      0.0000000      0.0000000"       # rx_twall(:,1) / dt
    assert lines[12] == "      0.0000000      0.0000000      0.0000000"       # rx_twall(:,2) / dt^2
    assert lines[13] == "            1            0           -2"             # pbc_twall
    assert lines[17] == "            0            0            1"             # s_force_grad
    assert lines[18] == "" and len(lines) == 19


def test_conf_round_trip(tmp_path, melt_cfg):
    cfg = melt_cfg
    path = str(tmp_path / "conf_new")
    a = np.random.default_rng(3).normal(size=(cfg.n, 3)) * 50.0
    checkpoint.write_conf(path, cfg.r0, cfg.v, a, cfg.a_type, cfg.params.n_mon, cfg.params.n_chain)
    st = checkpoint.read_conf(path, cfg.n)
    assert (st["n_mon"], st["n_chain"], st["n_order"]) == (cfg.params.n_mon, cfg.params.n_chain, 2)
    assert (st["a_type"] == cfg.a_type).all()
    # 7 decimals: half a unit in the last place
    assert np.abs(st["r0"] - cfg.r0).max() <= 5.0001e-8
    assert np.abs(st["v"] - cfg.v).max() <= 5.0001e-8
    assert np.abs(st["a"] - a).max() <= 5.0001e-8
    np.testing.assert_array_equal(st["walls"]["pbc_twall"], [0, 0, 0])


def test_conf_reader_rejects_a_short_file(tmp_path):
    path = tmp_path / "conf_old"
    path.write_text("1\n         2         1\n         0         0\n  2\n")
    with pytest.raises(ValueError):
        checkpoint.read_conf(str(path), 10)


def test_state_round_trip_is_exact(tmp_path, brush_small_cfg):
    cfg = brush_small_cfg
    rng = np.random.default_rng(4)
    a = rng.normal(size=(cfg.n, 3))
    mic = rng.integers(-3, 4, size=(cfg.n, 3)).astype(np.int32)
    path = str(tmp_path / "state.bin")
    checkpoint.write_state(path, cfg.r0, cfg.v, a, mic, cfg.a_type, 123456789)
    st = checkpoint.read_state(path)
    assert st["i_time"] == 123456789
    for name, ref in (("r0", cfg.r0), ("v", cfg.v), ("a", a)):
        assert st[name].tobytes() == np.ascontiguousarray(ref, dtype="<f8").tobytes(), name
    assert (st["mic"] == mic).all() and (st["a_type"] == cfg.a_type).all()
    raw = bytearray(open(path, "rb").read())
    raw[0] ^= 1
    open(path, "wb").write(bytes(raw))
    with pytest.raises(ValueError):
        checkpoint.read_state(path)


def test_oracle_resumes_from_the_side_car(tmp_path, melt_cfg):
    """A run stopped after 30 steps, written to the side-car and resumed (lists
    rebuilt from the loaded positions, as the start-up does) follows the
    uninterrupted run: the same positions up to the summation order of the
    rebuilt lists (thermostat off, FP64)."""
    cfg = melt_cfg
    p = cfg.params.copy()
    p.thermostat = _abi.THERMO_NONE
    o1 = Oracle(p, cfg.r0, cfg.v, cfg.a_type, cfg.mass)
    o1.init_forces()
    for _ in range(30):
        o1.md_step()
    s = o1.state()
    path = str(tmp_path / "state.bin")
    checkpoint.write_state(path, s["r0"], s["v"], s["a"], s["mic"], cfg.a_type, 30)
    st = checkpoint.read_state(path)
    o2 = Oracle(p, st["r0"], st["v"], st["a_type"], cfg.mass, a=st["a"], mic=st["mic"])
    o2.set_step(st["i_time"])
    o2.binning()
    for _ in range(20):
        o1.md_step()
        o2.md_step()
    assert np.abs(o1.state()["r0"] - o2.state()["r0"]).max() < 1e-10


@pytest.mark.gpu
def test_system_save_and_restore(tmp_path, brush_small_cfg):
    """The side-car moves a System's state into another System bit for bit
    (step counter included); both then run on alike (rounding of the rebuilt
    lists' summation order)."""
    from mfa_b200.api import System
    cfg = brush_small_cfg
    g1 = System(cfg.params, cfg.r0, cfg.v, cfg.a_type, cfg.mass, precision=FP64)
    g1.init_forces()
    g1.step(40)
    path = str(tmp_path / "state.bin")
    checkpoint.save(g1, conf_path=str(tmp_path / "conf_new"), state_path=path)
    g2 = System(cfg.params, cfg.r0, cfg.v, cfg.a_type, cfg.mass, precision=FP64)
    checkpoint.restore(g2, state_path=path)
    a, b = g1.download(), g2.download()
    for k in ("r0", "v", "a", "mic"):
        assert np.array_equal(a[k], b[k]), k
    assert g2.scalars()["i_time"] == 40
    g1.binning()              # the same rebuild point for both
    g1.step(20)
    g2.step(20)
    assert float(np.abs(g1.download()["r0"] - g2.download()["r0"]).max()) < 1e-11
    st = checkpoint.read_conf(str(tmp_path / "conf_new"), cfg.n)
    assert np.abs(st["r0"] - a["r0"]).max() <= 5.0001e-8
    g1.close()
    g2.close()
