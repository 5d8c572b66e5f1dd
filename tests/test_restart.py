"""Restart files in the reference's format (cJupiterModel::save_state / load_state,
FileIO_Jup.cpp:261-683): atjup_gpu_save_state / atjup_gpu_load_state.

* A file the reference writes after two full-physics iterations loads onto the GPU with every
  array bit-identical to the reference's at that point, and the GPU run resumed from it follows the
  reference's own iterations 3 and 4 within the bars of the full-physics step (tests/
  test_moist_step.py).
* A file the GPU writes loads into the reference with its own load_state, every restart array
  bit-identical to the GPU's (thermalmassflux, which the device path does not compute, as zeros).
* GPU save, load into a fresh context and resume is bit-identical to the straight GPU run with
  carried = 2 (JUP2 plus a trailer of the five arrays the next iterations read when they are
  non-zero and the reference's list omits); the plain JUP2 and JUP1 files have exactly the
  reference's layout and size.
* Bad files are refused before the device state is touched."""
import struct
import tempfile
from pathlib import Path

import numpy as np
import pytest

from helpers import ref_dump, synthetic_case
from moist_cases import PROGNOSTIC, gpu_moist_model, ref_iters_case, synthetic_moist_case
from oracle_bridge import rel_l2
from test_moist_step import NH4SH_FAMILY_TOL, REF_TOL

# the reference's restart arrays the device holds, by device name; the n copies of the scalars
# are compared through download_n, t/u/v/w/p_dyn n copies equal the live fields between steps
LIVE = ("t", "u", "v", "w", "p_dyn", "p_stat", "nue", "aux_u", "aux_v", "aux_w", "difflux_h2s",
        "difflux_nh3", "massflux_h2s", "massflux_nh3", "fluxlim_nh4sh", "Q_precip", "Q_rad",
        "rho_mix", "S_precip_h2o", "S_precip_h2o_cloud", "S_precip_h2o_ice", "S_precip_nh3",
        "S_precip_nh3_ice", "h2o", "h2o_cloud", "h2o_ice", "h2s", "nh3", "nh3_cloud", "nh3_ice",
        "ch4", "ch4_cloud", "ch4_ice", "nh4sh", "tke", "dis")
NCOPIES = ("h2o", "h2o_cloud", "h2o_ice", "h2s", "nh3", "nh3_cloud", "nh3_ice", "ch4",
           "ch4_cloud", "ch4_ice", "nh4sh", "tke", "dis")
JUP1, JUP2 = 0x4A555031, 0x4A555032


def assert_same(name, got, want):
    assert np.array_equal(got, want, equal_nan=True), \
        f"{name}: differs (max |d| {np.nanmax(np.abs(got - want)):.3e})"


@pytest.mark.gpu
def test_reference_restart_resumes_on_gpu(ref_required):
    tmp = tempfile.mkdtemp(prefix="atjup_rs_")
    d, P, PH, MC, g, f = ref_iters_case(4, "--save-restart", f"{tmp}:2")
    m = gpu_moist_model(P, PH, MC, g, f)
    it, carried = m.load_state(Path(tmp) / "jup_restart_2.bin")
    assert (it, carried) == (2, 1)
    for n in LIVE:
        assert_same(n, m.download(n), d[f"rs2_{n}"])
    for n in NCOPIES:
        assert_same(n + "n", m.download_n(n), d[f"rs2_{n}n"])
    assert_same("vel_star", m.download2d("vel_star"), d["rs2_vel_star"])
    for it in (3, 4):
        m.step(it, first=False)
    for n in PROGNOSTIC:
        r = rel_l2(m.download(n), d[f"it4_{n}"])
        assert r <= NH4SH_FAMILY_TOL.get(n, REF_TOL), f"resumed iteration 4: {n} relative L2 {r:.3e}"
    m.close()


@pytest.mark.gpu
def test_gpu_restart_loads_in_reference(ref_required):
    d, P, PH, MC, g, f = ref_iters_case(3)
    m = gpu_moist_model(P, PH, MC, g, f)
    for it in (1, 2):
        m.step(it, first=(it == 1))
    tmp = tempfile.mkdtemp(prefix="atjup_rs_")
    m.save_state(Path(tmp) / "jup_restart_2.bin", 2)
    r = ref_dump("--load-restart", f"{tmp}:2")
    assert int(r["load_rc"]) == 0
    for n in LIVE:
        assert_same(n, r[f"rs_{n}"], m.download(n))
    for n in NCOPIES:
        assert_same(n + "n", r[f"rs_{n}n"], m.download_n(n))
    for n, live in (("tn", "t"), ("un", "u"), ("vn", "v"), ("wn", "w"), ("p_dynn", "p_dyn")):
        assert_same(n, r[f"rs_{n}"], m.download(live))
    assert not np.any(r["rs_thermalmassflux"])
    assert_same("vel_star", r["rs_vel_star"], m.download2d("vel_star"))
    m.close()


@pytest.mark.gpu
def test_gpu_save_load_resume_is_bit_identical():
    P, PH, MC, g, f = synthetic_moist_case(13, 37, 49, seed=47)
    straight = gpu_moist_model(P, PH, MC, g, f)
    first = gpu_moist_model(P, PH, MC, g, f)
    for it in (1, 2):
        straight.step(it, first=(it == 1))
        first.step(it, first=(it == 1))
    tmp = Path(tempfile.mkdtemp(prefix="atjup_rs_"))
    first.save_state(tmp / "jup2.bin", 2)
    first.save_state(tmp / "jup1.bin", 2, carried=0)
    first.save_state(tmp / "jup2x.bin", 2, carried=2)
    first.close()
    im, jm, km = P.im, P.jm, P.km
    n3 = im * jm * km * 8
    hdr2 = struct.unpack("<5i", (tmp / "jup2.bin").read_bytes()[:20])
    assert hdr2 == (JUP2, im, jm, km, 2)
    assert (tmp / "jup2.bin").stat().st_size == 20 + (38 + 17) * n3 + jm * km * 8
    assert struct.unpack("<i", (tmp / "jup1.bin").read_bytes()[:4])[0] == JUP1
    assert (tmp / "jup1.bin").stat().st_size == 20 + 38 * n3
    assert (tmp / "jup2x.bin").stat().st_size == 20 + (38 + 17) * n3 + jm * km * 8 + 8 + 5 * n3
    # a fresh context from the initial state, as the reference's resume starts from its own
    # initialisation; the file then replaces every array the next iterations read
    resumed = gpu_moist_model(P, PH, MC, g, f)
    assert resumed.load_state(tmp / "jup2x.bin") == (2, 2)
    for it in (3, 4):
        straight.step(it, first=False)
        resumed.step(it, first=False)
    for n in PROGNOSTIC + ("Q_rad", "Q_precip", "rho_mix", "aux_u", "nue"):
        assert_same(n, resumed.download(n), straight.download(n))
    for n in NCOPIES:
        assert_same(n + "n", resumed.download_n(n), straight.download_n(n))
    straight.close()
    resumed.close()


@pytest.mark.gpu
def test_load_refuses_bad_files():
    from atjup_b200.gpu import AtjupError, GpuModel
    P, g, f = synthetic_case(13, 37, 49, seed=5)
    m = GpuModel(P, g)
    m.upload_state(f)
    tmp = Path(tempfile.mkdtemp(prefix="atjup_rs_"))
    m.save_state(tmp / "good.bin", 7)
    raw = (tmp / "good.bin").read_bytes()
    (tmp / "short.bin").write_bytes(raw[: len(raw) // 2])
    (tmp / "magic.bin").write_bytes(struct.pack("<i", 0x12345678) + raw[4:])
    P2, g2, _ = synthetic_case(13, 37, 33, seed=5)
    other = GpuModel(P2, g2)
    t_before = m.download("t")
    for name in ("short.bin", "magic.bin", "missing.bin"):
        with pytest.raises(AtjupError):
            m.load_state(tmp / name)
    with pytest.raises(AtjupError):
        other.load_state(tmp / "good.bin")            # grid mismatch
    assert_same("t", m.download("t"), t_before)       # refused before the device was touched
    assert m.load_state(tmp / "good.bin") == (7, 1)
    m.close()
    other.close()
