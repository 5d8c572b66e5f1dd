"""Host-side tests (no GPU): the C ABI library loads and exports every declared entry point,
its default parameter block matches the host knob resolution, knobs map to the reference's
branches, the replica timing aggregation works over a 2-rank gloo group."""
import ctypes
import os
import re
from pathlib import Path

import pytest

from atjup_b200 import params as P

ROOT = Path(__file__).resolve().parents[1]
LIB = ROOT / "atjup_b200" / "libatjup_gpu.so"


def declared_entry_points():
    src = (ROOT / "include" / "atjup_gpu.h").read_text()
    return sorted(set(re.findall(r"\b(atjup_(?:gpu|params)_\w+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    if not LIB.exists():
        pytest.skip("libatjup_gpu.so not built")
    return ctypes.CDLL(str(LIB))


def test_library_exports_every_declared_entry_point(lib):
    names = declared_entry_points()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_default_params_match_host_resolution(lib):
    c = P.AtjupParams()
    lib.atjup_params_default(ctypes.byref(c))
    h = P.resolve_params({})
    for name, _ in P._FIELDS:
        a, b = getattr(c, name), getattr(h, name)
        assert a == pytest.approx(b, rel=1e-15, abs=0), name


def test_params_struct_size_matches_oracle():
    from oracle_bridge import build_oracle
    so = ctypes.CDLL(str(build_oracle()))
    so.ora_params_sizeof.restype = ctypes.c_size_t
    assert so.ora_params_sizeof() == ctypes.sizeof(P.AtjupParams)
    so.ora_gas_params_sizeof.restype = ctypes.c_size_t
    assert so.ora_gas_params_sizeof() == ctypes.sizeof(P.AtjupGasParams)
    so.ora_micro_sizeof.restype = ctypes.c_size_t
    assert so.ora_micro_sizeof() == ctypes.sizeof(P.AtjupMicro)
    so.ora_sat_stats_sizeof.restype = ctypes.c_size_t
    assert so.ora_sat_stats_sizeof() == ctypes.sizeof(P.AtjupSatStats)


def test_create_without_device_reports_no_device(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    p = P.resolve_params({})
    ctx = ctypes.c_void_p()
    rc = lib.atjup_gpu_create(ctypes.byref(p), ctypes.byref(ctx))
    assert rc == 6 and not ctx.value


def test_knob_resolution_follows_reference_defaults():
    p = P.resolve_params({})
    assert p.nd_cor == pytest.approx(1400.0)          # ATJUP_ND_COR follows geo balance
    assert p.metric_split == 1 and p.coriolis_split == 1 and p.hydro_split == 0
    assert p.cell_hold == 1 and p.rho_pdyn == 0 and p.v_massbal_zonal == 1
    assert p.p_dyn_to_bar == pytest.approx(1.2844 * 100.0 ** 2 * 1e-5)
    q = P.resolve_params({"ATJUP_GEO_BALANCE": "0", "ATJUP_NONDIM": "1"})
    assert q.nd_cor == pytest.approx(1400.0) and q.nd_buoy == pytest.approx(1.4e6)
    assert q.hydro_split == 1 and q.cell_hold == 0 and q.rho_pdyn == 1
    assert P.resolve_params({"ATJUP_BUOY_RAMP_ITERS": "10"}, iter_n=4).buoy_ramp == pytest.approx(0.4)
    assert P.resolve_params({"ATJUP_PRESS_SWEEPS": "0"}).press_sweeps == 1


def test_unsupported_knobs_are_named():
    assert P.check_supported({}) == []
    bad = P.check_supported({"ATJUP_PRESS_LINE": "1", "ATJUP_T_LIMITER": "0"})
    assert len(bad) == 1 and bad[0].startswith("ATJUP_PRESS_LINE=1")
    # NH4SH by the rate law is implemented in its default form only
    assert P.check_supported({"ATJUP_NH4SH_EQ": "0"}) == []
    bad = P.check_supported({"ATJUP_NH4SH_EQ": "0", "ATJUP_CHEM_MOLAR_CONC": "1",
                             "ATJUP_CHEM_GATE_ZERO": "0"})
    assert sorted(b.split("=")[0] for b in bad) == ["ATJUP_CHEM_GATE_ZERO", "ATJUP_CHEM_MOLAR_CONC"]
    mc = P.resolve_micro({"ATJUP_NH4SH_EQ": "0"})
    assert mc.nh4sh_eq == 0 and (mc.t_0_nh4sh, mc.t_00_nh4sh) == (230.0, 200.0)


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    from atjup_b200.replicas import max_over_ranks, whole_job_seconds_per_step
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    m = max_over_ranks(1.5 + rank)                      # rank 1 is the slow one
    out[rank] = (m, whole_job_seconds_per_step(m, 10, world))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_timing_is_max_over_ranks():
    import socket

    import torch.multiprocessing as mp
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    with mp.get_context("spawn").Manager() as mgr:   # no fork of a process that may hold a GPU
        out = mgr.dict()
        mp.spawn(_rank_main, args=(2, port, out), nprocs=2, join=True)
        assert out[0] == out[1] == (2.5, 2.5 / 20)


def test_field_ids_match_the_header():
    """The Python field ids (atjup_b200.params) are the header's enum, in order (the Python names
    are the reference's array names: compared without case and underscores)."""
    src = (ROOT / "include" / "atjup_gpu.h").read_text()
    body = src[src.index("ATJUP_F_T = 0"):src.index("ATJUP_F_COUNT")]
    names = re.findall(r"ATJUP_F_(\w+)", body)
    py = {v: k for k, v in P.FIELD_IDS.items()}
    assert len(names) == len(P.FIELD_IDS)
    for i, n in enumerate(names):
        assert py[i].lower().replace("_", "") == n.lower().replace("_", ""), (i, n, py[i])
    s_body = src[src.index("ATJUP_S_H2O = 0"):src.index("ATJUP_S_COUNT")]
    assert [x.lower() for x in re.findall(r"ATJUP_S_(\w+)", s_body)] == list(P.SPECIES)
