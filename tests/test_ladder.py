"""A temperature ladder split over ranks (tis_b200.remd, the library's
tis_rex_decide), on CPU with gloo ranks and the oracle standing in for each
rank's GPU context.

A 16-replica ladder split 8 + 8 over two ranks, with identical injected
noise and uniforms, gives the same labels, accept counts and velocities as
the single-process oracle run (oracle/: orc_replica_exchange, the
restatement of energy_allrep + simu_replica_exchange) over two exchanges,
one of each odd/even alternation.  Each rank's oracle steps the whole ladder
(the same numbers on both ranks) but contributes only its own replicas'
energies; the gathered energies and the library's host decision then drive
every rank.
"""
import ctypes as C
import os
import socket

import numpy as np
import pytest

from tis_b200 import remd, synth

NREP, NSTEP = 16, 12


def test_ladder_share():
    assert remd.ladder_share(16, 2, 0) == (1, 8) and remd.ladder_share(16, 2, 1) == (9, 8)
    shares = [remd.ladder_share(10, 4, r) for r in range(4)]
    assert shares == [(1, 3), (4, 3), (7, 2), (9, 2)]
    with pytest.raises(ValueError):
        remd.ladder_share(2, 4, 0)


def _system():
    s = synth.set_friction(synth.dt15_chain(22, 1, stem=6), 0.5)
    return synth.hairpin_coords(s, 6, seed=1)


def _noise(k, n):
    return np.random.default_rng(100 + k).normal(size=(NSTEP + (1 if k == 0 else 0), NREP, n, 3))


def _uniforms(k):
    return np.random.default_rng(200 + k).uniform(size=NREP)


def _run_single():
    from oracle.oracle import Oracle
    s = _system()
    ladder = synth.temperature_ladder(NREP, 280.0, 400.0)
    par = synth.dt15_params(ionic_strength=0.15, precision=0)
    orc = Oracle(s, par, ladder)
    orc.set_state(np.tile(s["xyz"], (NREP, 1, 1)))
    out = []
    for k in range(2):
        orc.set_noise(_noise(k, s["nmp"]))
        if k == 0:
            orc.time_integral_pre()
        orc.step(NSTEP)
        nacc = orc.replica_exchange(_uniforms(k))
        out.append((orc.labels().copy(), orc.get_state()[1].copy(), nacc))
    return out


def _rank_main(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    from oracle.oracle import Oracle
    from tis_b200.abi import load_library, ptr_f64, ptr_i32
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        lib = load_library()          # the host decision needs no GPU
        s = _system()
        ladder = np.array(synth.temperature_ladder(NREP, 280.0, 400.0))
        par = synth.dt15_params(ionic_strength=0.15, precision=0)
        orc = Oracle(s, par, list(ladder))
        orc.set_state(np.tile(s["xyz"], (NREP, 1, 1)))
        first, count = remd.ladder_share(NREP, world, rank)
        out = []
        idx_pair = 1
        for k in range(2):
            orc.set_noise(_noise(k, s["nmp"]))
            if k == 0:
                orc.time_integral_pre()
            orc.step(NSTEP)
            local = np.array([orc.replica_energy(first + i) for i in range(count)])
            e_all = remd.gather_energies(local, NREP, dist, "cpu")
            r2l = np.ascontiguousarray(orc.labels(), dtype=np.int32)
            vs = np.zeros(NREP)
            nacc = C.c_int32(0)
            u = np.ascontiguousarray(_uniforms(k))
            e = np.ascontiguousarray(e_all)
            rc = lib.tis_rex_decide(NREP, ptr_f64(ladder), idx_pair, ptr_f64(e), ptr_f64(u), ptr_i32(r2l),
                                    ptr_f64(vs), C.byref(nacc))
            assert rc == 0
            orc.rex_apply(r2l, vs)
            idx_pair = 2 if idx_pair == 1 else 1
            v = orc.get_state()[1]
            out.append((r2l.copy(), v[first - 1:first - 1 + count].copy(), nacc.value))
        q.put((rank, first, count, out))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_ladder_split_gloo_world2_matches_single_process():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in range(2)]
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    single = _run_single()
    assert any(n > 0 for _, _, n in single)         # some swaps happen
    for rank, first, count, out in res:
        for (lab, v, nacc), (lab1, v1, nacc1) in zip(out, single):
            assert nacc == nacc1
            assert np.array_equal(lab, lab1)
            assert np.array_equal(v, v1[first - 1:first - 1 + count])
