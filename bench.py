#!/usr/bin/env python
"""Throughput of the QG core on B200: Mcell-layer-steps/s.

Default workload (N=1): the ocean basin of the coupled configuration, a
513 x 513 p-point, 3-layer double-gyre box at dx = 10 km in FP64, stepped
with tdt = 2 dt = 3600 s.  One bench step is a batch of 10 model steps (the
configuration's 10 ocean steps); Mcell-layer-steps/s counts
nxp * nyp * nl * model steps / s / 1e6, summed over ranks.

  value   device time of the batches (CUDA events on the handle's stream),
          inputs resident in HBM, L2 flushed (a 256 MiB write) before every
          timed batch;
  e2e     the same work through the C ABI with host buffers: per model step
          the coupler's exchange of driver.F90:99-107 -- forcing (wekp, ent)
          uploaded from pinned host memory, one step, layer-1 pressure read
          back -- timed by the host clock;
  roofline  the dominant kernel (largest share of a step), timed alone by
          oqg_profile_phases, against the measured HBM copy bandwidth;
  cpu_baseline  the FP64 oracle (a restatement of the reference's Fortran,
          one thread) on a bounded sample of the same basin.

--impl reference times the CPU restatement of the reference (the oracle,
all host threads) on the same workload; the Fortran reference itself does
not build here (no Fortran compiler, FFTW, LAPACK or netCDF).

Multi-GPU (torchrun): every rank steps its own basin (replicas, weak
scaling); the time is the max over ranks.
"""
import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # name: (builder kwargs, tdt, label)
    "ocean513": (dict(kind="box", n=513, dx=10e3), 3600.0,
                 "ocean double gyre 513x513x3 box, dx 10 km (coupled config ocean basin)"),
    "ocean129": (dict(kind="box", n=129, dx=20e3), 3600.0,
                 "ocean double gyre 129x129x3 box, dx 20 km"),
    "atmos193x97": (dict(kind="channel", nxp=193, nyp=97, dx=80e3), 360.0,
                    "atmosphere channel 193x97x3, dx 80 km (coupled config atmosphere)"),
    "ocean1025": (dict(kind="box", n=1025, dx=10e3), 3600.0,
                  "ocean double gyre 1025x1025x3 box, dx 10 km"),
    "ocean2049": (dict(kind="box", n=2049, dx=5e3, ah4=1e9), 1200.0,
                  "eddy-resolving ocean 2049x2049x3 box, dx 5 km, ah4 1e9, dt 600 s"),
}


def make_basin(name, precision):
    from openqg_b200.params import atmos_channel, ocean_double_gyre
    kw, tdt, label = WORKLOADS[name]
    if kw["kind"] == "box":
        b = ocean_double_gyre(kw["n"], dx=kw["dx"], ah4=kw.get("ah4", 2.0e10), precision=precision)
    else:
        b = atmos_channel(kw["nxp"], kw["nyp"], dx=kw["dx"], precision=precision)
    return b, tdt, label


ENSEMBLE_SIZES = (65, 97, 129, 193, 257)


def make_ensemble(precision, members=256, seed=0):
    """The batched-ensemble configuration: square 3-layer ocean basins at
    dx = 20 km with sizes drawn uniformly from ENSEMBLE_SIZES; per member a
    wind amplitude in [0.05, 0.15] N/m^2, ah4 in [1e10, 4e10] m^4/s and its
    own seeded initial stream function (std 1e3 m^2/s)."""
    from openqg_b200.core import ekman_from_tau
    from openqg_b200.params import double_gyre_tau, initial_psi, ocean_double_gyre
    rng = np.random.default_rng(seed)
    sizes = rng.choice(ENSEMBLE_SIZES, size=members)
    amps = rng.uniform(0.05, 0.15, size=members)
    ah4s = rng.uniform(1e10, 4e10, size=members)
    basins, inputs = [], []
    for i in range(members):
        b = ocean_double_gyre(int(sizes[i]), dx=20e3, ah4=float(ah4s[i]), precision=precision)
        p = b.fnot * initial_psi(b, seed=1000 + i)
        w, ts, tn = ekman_from_tau(b, *double_gyre_tau(b, amp=float(amps[i])))
        basins.append(b)
        inputs.append((p, w, ts, tn))
    return basins, inputs


def ensemble_shard(n, rank, ws):
    """The members rank steps when ws ranks share an ensemble of n: every
    ws-th member from rank (the sizes are drawn independently, so each rank
    gets a like mix)."""
    return list(range(rank, n, ws))


def run_ensemble(precision, steps, warmup, msteps, flush, tdt=3600.0, rank=0, ws=1):
    """The ensemble's steps on this rank, one launch per phase: its shard of
    the members (ensemble_shard), so ws ranks together step the whole
    ensemble once.  Returns the cell-layers of the whole ensemble, this
    rank's time and the tile height."""
    import torch
    from openqg_b200.core import Ensemble
    all_basins, all_inputs = make_ensemble(precision)
    mine = ensemble_shard(len(all_basins), rank, ws)
    basins, inputs = [all_basins[i] for i in mine], [all_inputs[i] for i in mine]
    e = Ensemble(basins)
    for i, (p, w, ts, tn) in enumerate(inputs):
        e.set_state(i, p, p)
        e.set_forcing(i, w, None, ts, tn)
    # one vorticity tile height for all members, measured (oqg_ensemble_autotune)
    tile_rows, _ = e.autotune(tdt, 4)
    for _ in range(warmup):
        e.step(tdt, msteps)
    e.sync()
    s = torch.cuda.ExternalStream(e.stream())
    total = 0.0
    torch.cuda.nvtx.range_push("ensemble_steps")
    for _ in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        e.step(tdt, msteps)
        e1.record(s)
        e1.synchronize()
        total += e0.elapsed_time(e1)
    torch.cuda.nvtx.range_pop()
    e.sync()
    cells = sum(b.nxp * b.nyp * b.nl for b in all_basins)
    e.close()
    return cells, total, tile_rows


# box sizes of the adjoint runs: n -> (dx, ah4, tdt)
ADJOINT_BOXES = {257: (20e3, 2.0e10, 3600.0), 1025: (5e3, 1.0e9, 1200.0), 2049: (5e3, 1.0e9, 1200.0)}


def run_adjoint(reps=3, n=257, dx=20e3, ah4=2.0e10, nsteps=200, every=20, tdt=3600.0):
    """The differentiable configuration (default: 3-layer ocean box at
    257x257, dx 20 km, 200 leapfrog steps, checkpoint every 20 steps with
    recomputation), J = ekei(1) of the final state, gradients with respect to
    the initial stream function and the wind forcing.  Device times between
    CUDA events on the handle's stream (host waits inside a pass included) of
    the plain forward run, the checkpointed forward, the reverse pass
    (recompute + adjoint) and nsteps adjoint steps alone; medians over reps
    after one untimed repetition."""
    import torch
    from openqg_b200.adjoint import AdjointRun, ekei
    from openqg_b200.core import QG, lib
    from openqg_b200.params import ocean_double_gyre
    b = ocean_double_gyre(n, dx=dx, ah4=ah4)
    p, w, ts, tn = initial_inputs(b, seed=5)
    g = QG(b)
    g.set_forcing(w, None, ts, tn)
    s = torch.cuda.ExternalStream(g.stream())

    def timed(fn):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        fn()
        e1.record(s)
        e1.synchronize()
        return e0.elapsed_time(e1)

    run = AdjointRun(g, every)
    L = lib()
    slot = ctypes.c_void_p(run.slots[0].data_ptr())
    fwd, ck, bwd, adj = [], [], [], []
    gnorm = 0.0
    for _ in range(reps + 1):
        g.set_state(p, p)
        g.set_step_index(0)
        fwd.append(timed(lambda: g.step(tdt, nsteps)))
        g.set_state(p, p)
        g.set_step_index(0)
        ck.append(timed(lambda: run.forward(nsteps, tdt)))
        pf = torch.as_tensor(g.get_state()[0], device="cuda").requires_grad_(True)
        (gp,) = torch.autograd.grad(ekei(b, pf)[0], [pf])
        out = {}
        bwd.append(timed(lambda: out.update(run.backward(lp=gp))))
        gnorm = float(out["gp0"].norm()) + float(out["lwekp"].norm())
        L.oqg_pq_save(g.h, slot)

        def adj_only():
            # an NVTX range marks these launches for a profiler's filter
            torch.cuda.nvtx.range_push("adjoint_steps")
            for i in range(nsteps):
                L.oqg_adj_step(g.h, slot, ctypes.c_double(tdt), ctypes.c_longlong(2 + i % 20))
            torch.cuda.nvtx.range_pop()

        adj.append(timed(adj_only))
    g.close()
    med = lambda x: statistics.median(x[1:]) / nsteps
    if not math.isfinite(gnorm):
        raise RuntimeError("non-finite adjoint gradient")
    f, c, r, a = med(fwd), med(ck), med(bwd), med(adj)
    return {"workload": "ocean %dx%dx3 box, dx %g km, ah4 %g, tdt %g s, %d steps, checkpoint every %d, "
                        "J = ekei(1), gradient w.r.t. initial psi and wind forcing"
                        % (n, n, dx / 1e3, ah4, tdt, nsteps, every),
            "forward_ms_per_step": f, "checkpointed_forward_ms_per_step": c,
            "reverse_ms_per_step": r, "adjoint_step_ms": a,
            "reverse_over_forward": r / f, "adjoint_step_over_forward_step": a / f,
            "launches_per_adjoint_step": "5 (6 when a suppression is transposed)",
            "timer": "CUDA events on the handle's stream, median of %d runs" % reps}


def coupled_e2e(g, b, tdt, msteps, nbatch):
    """The ocean step of the coupled driver (driver.F90:95-107) with the mixed
    layer on the device: per model step the wind stress (taux, tauy at p
    points) and the net heat flux (T points) cross from pinned host memory,
    oqg_ocean_forcing runs ekman_from_tau and step_oml into the handle's
    forcing, and step_qg runs; p(:,:,1) and ent stay on the device.  Host
    clock, median over nbatch batches of msteps model steps."""
    import torch
    from openqg_b200.core import OceanMixedLayer, lib
    from openqg_b200.params import double_gyre_tau
    L = lib()
    taux, tauy = double_gyre_tau(b)
    nyt, nxt = b.nyp - 1, b.nxp - 1
    yy = np.linspace(0.0, 1.0, nyt)[:, None]
    sst = 12.0 + 3.0 * np.cos(np.pi * yy) * np.ones((1, nxt))
    m = OceanMixedLayer(g, hm=100.0, rho_cp=4.0e6, t1_rel=10.0, dt_12=5.0, st2d=2.0e3, st4d=0.0, ycexp=1.0)
    m.set_sst(sst, sst)
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).pin_memory()
    tx, ty = pin(taux), pin(tauy)
    fn = pin(20.0 * np.cos(np.pi * yy) * np.ones((1, nxt)))
    args = [ctypes.c_void_p(t.data_ptr()) for t in (tx, ty, fn)]

    def batch():
        for _ in range(msteps):
            rc = L.oqg_ocean_forcing(m.h, *args, 1, ctypes.c_double(tdt))
            rc |= L.oqg_step(g.h, ctypes.c_double(tdt), 1)
            if rc:
                raise RuntimeError(L.oqg_last_error().decode())
        g.sync()

    batch()
    times = []
    torch.cuda.nvtx.range_push("ocean_forcing")
    for _ in range(nbatch):
        t0 = time.perf_counter()
        batch()
        times.append((time.perf_counter() - t0) * 1e3)
    torch.cuda.nvtx.range_pop()
    m.close()
    ms = statistics.median(times)
    cells = b.nxp * b.nyp * b.nl
    return {"value": cells * msteps / (ms / 1e3) / 1e6, "unit": "Mcell-layer-steps/s",
            "h2d_bytes_per_step": msteps * (2 * b.nxp * b.nyp + nxt * nyt) * 8, "d2h_bytes_per_step": 0,
            "pattern": "per model step: upload taux, tauy, fnetoc; ekman + ocean mixed layer + step on the "
                       "device (p(:,:,1), wekp and ent stay there)",
            "timer": "host clock, median of %d steps" % nbatch}


def coupled_config(nrep=3, nocean=10, nstr=10, precision=None):
    """The coupled configuration's step loop on the device (dynamic_step,
    driver.F90:33-143): per ocean step, xforc (both basins' wind stress from
    the atmosphere's lagged pressure, the ocean's through the bicubic
    interpolation) and compute_forcing (both mixed layers' net heat fluxes),
    then nstr atmosphere steps (193x97x3 channel, dx 80 km, tdt 360 s) each
    after oqg_atmos_forcing, the first followed by one ocean step (513x513x3
    box, dx 10 km, tdt 3600 s) after oqg_ocean_forcing.  Every exchange runs
    on the device; nothing crosses from the host inside the loop.  The
    radiation and mixed-layer parameters are the reference's coupled
    double-gyre configuration's (data/basin/atm_dg.cdl, ocn_dg.cdl) through
    the radiative start-up (oqg_radiat and its helpers); the mixed layers
    start from the radiative-balance profiles (rbal) with seeded SST noise
    (std 0.5 K), the QG states from seeded noise.  precision OQG_MIXED: both
    handles store their state in FP32 (the configuration's FP32-bulk form).  Host clock over nocean
    coupled ocean steps, median of nrep."""
    from openqg_b200.core import QG, AtmosMixedLayer, OceanMixedLayer, lib
    from openqg_b200.params import OQG_FP64, atmos_channel, ocean_double_gyre
    from openqg_b200.radiation import coupled_start, rbal_states
    L = lib()
    prec = OQG_FP64 if precision is None else precision
    bo, ba = ocean_double_gyre(513, dx=10e3, precision=prec), atmos_channel(193, 97, dx=80e3, precision=prec)
    rad, ak, ok = coupled_start(ba, bo, hm_a=1000.0, fsbar=-210.0, fspamp=80.0, zopt=[200.0, 3.0e4, 3.0e4, 4.0e4],
                                gamma=1.0e-2, xlamda=35.0, tabsat=[330.0, 340.0, 350.0], rho_a=1.0, cp_a=1.0e3,
                                t1_abs_o=278.0, t2_abs_o=268.0, rho_o=1.0e3, cp_o=4.0e3)
    go, ga = QG(bo), QG(ba)
    po, _, _, _ = initial_inputs(bo, seed=3)
    pa, _, _, _ = initial_inputs(ba, seed=4)
    go.set_state(po, po)
    ga.set_state(pa, pa)
    oml = OceanMixedLayer(go, hm=100.0, rho_cp=ok["rho_cp"], t1_rel=ok["t1_rel"], dt_12=ok["dt_12"], st2d=380.0,
                          st4d=4.0e10, ycexp=1.0, fluxs=True, sval=ok["sval"], nval=ok["nval"])
    _, sst, ast = rbal_states(ba, bo, rad, ak)
    sst = sst + 0.5 * np.random.default_rng(5).standard_normal(sst.shape)
    oml.set_sst(sst, sst)
    xc = ak["xc1ast"]
    aml = AtmosMixedLayer(ga, xc, None, hm=1000.0, rho_cp=ak["rho_cp"], t1_rel=ak["t1_rel"], dt_12=ak["dt_12"],
                          hmamin=100.0, hmadmp=0.15, xcexp=1.0, at2d=5.0e4, at4d=3.0e14, ahmd=2.0e5,
                          aface=ak["aface"], bface=ak["bface"], dface=ak["dface"], cdat=1.3e-3)
    aml.set_state(ast, ast, np.full(xc.shape, 1000.0), np.full(xc.shape, 1000.0))
    oml.couple(aml, 1.0e-3)     # rho_a / rho_o
    rad = rad.c

    def coupled_step():
        rc = L.oqg_xforc(aml.h, oml.h)
        rc |= L.oqg_compute_forcing(oml.h, ctypes.byref(rad))
        for s in range(nstr):
            rc |= L.oqg_atmos_forcing(aml.h, None, None, None, 1, ctypes.c_double(360.0))
            rc |= L.oqg_step(ga.h, ctypes.c_double(360.0), 1)
            if s == 0:
                rc |= L.oqg_ocean_forcing(oml.h, None, None, None, 1, ctypes.c_double(3600.0))
                rc |= L.oqg_step(go.h, ctypes.c_double(3600.0), 1)
            if rc:
                raise RuntimeError(L.oqg_last_error().decode())

    coupled_step()
    go.sync()
    ga.sync()
    # each basin's tunable settings, measured on its own steps after the
    # first coupled step set its forcing (the states are restored)
    tuned = {}
    for name, g, tdt_g in (("ocean", go, 3600.0), ("atmosphere", ga, 360.0)):
        rows, _ = g.autotune(tdt_g, 10)
        yw, _ = g.autotune_ysolve(tdt_g, 10)
        xs, _ = g.autotune_xinv(tdt_g, 10)
        tuned[name] = {"tile_rows": rows, "ysolve_warps": yw, "xinv_two_launches": xs}
    times = []
    for _ in range(nrep):
        t0 = time.perf_counter()
        for _ in range(nocean):
            coupled_step()
        go.sync()
        ga.sync()
        times.append((time.perf_counter() - t0) * 1e3)
    if go.check_finite() or ga.check_finite():
        raise RuntimeError("non-finite state in the coupled run")
    oml.close()
    aml.close()
    go.close()
    ga.close()
    ms = statistics.median(times) / nocean
    cells = bo.nxp * bo.nyp * bo.nl + nstr * ba.nxp * ba.nyp * ba.nl
    return {"workload": "ocean 513x513x3 box (dx 10 km, tdt 3600 s) + atmosphere 193x97x3 channel (dx 80 km, "
                        "tdt 360 s, %d steps per ocean step); xforc (both stresses, bicubic onto the ocean), "
                        "compute_forcing (both heat fluxes), both mixed layers and Ekman fields on the device, "
                        "nothing from the host in the loop" % nstr,
            "state_storage": "fp32" if prec != OQG_FP64 else "fp64",
            "ms_per_coupled_ocean_step": ms, "value": cells / (ms / 1e3) / 1e6, "unit": "Mcell-layer-steps/s",
            "tuned": tuned,
            "timer": "host clock, median of %d runs of %d coupled ocean steps" % (nrep, nocean)}


def initial_inputs(b, seed, reference=False):
    """Seeded initial pressure and the double-gyre Ekman pumping.  The
    reference arm computes the pumping with the CPU restatement."""
    if reference:
        from oracle import ekman_from_tau
    else:
        from openqg_b200.core import ekman_from_tau
    from openqg_b200.params import double_gyre_tau, initial_psi
    p = b.fnot * initial_psi(b, seed=seed) * (30.0 if b.cyclic else 1.0)
    taux, tauy = double_gyre_tau(b)
    w, ts, tn = ekman_from_tau(b, taux, tauy)
    return p, w, ts, tn


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def traffic_table():
    """Bytes per launch from committed ncu summaries (profiles/traffic.txt)."""
    out = {}
    path = os.path.join(ROOT, "profiles", "traffic.txt")
    if os.path.exists(path):
        for line in open(path):
            f = line.split()
            if len(f) >= 4 and not line.startswith("#"):
                out[(f[0], f[1], f[2])] = float(f[3])
    return out


class Clocks:
    """nvidia-smi samples during the timed region."""

    def __init__(self, uuid):
        self.uuid = uuid
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap,"
             "clocks.mem,pstate")
        cmd = ["nvidia-smi", "--query-gpu=" + q, "--format=csv,noheader,nounits", "-lms", "200"]
        if self.uuid:
            cmd += ["-i", self.uuid]
        # compute processes on this GPU besides this one (a shared GPU slows the step)
        self.others = None
        try:
            qa = ["nvidia-smi", "--query-compute-apps=pid", "--format=csv,noheader"]
            if self.uuid:
                qa += ["-i", self.uuid]
            pids = subprocess.run(qa, capture_output=True, text=True, timeout=10).stdout.split()
            self.others = len([x for x in pids if x.strip().isdigit() and int(x) != os.getpid()])
        except Exception:
            pass
        try:
            self.proc = subprocess.Popen(cmd, stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) >= 9 and f[1].replace(".", "").isdigit():
                    rows.append(f)
        except Exception:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        mem = [float(r[9]) for r in rows if len(r) > 9 and r[9].replace(".", "").isdigit()]
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][2]),
                "mem_mhz": statistics.median(mem) if mem else None,
                "pstates": sorted({r[10] for r in rows if len(r) > 10}),
                "reasons": reasons, "samples": len(rows), "other_processes": self.others}


def cpu_sample(b, p, w, ts, tn, tdt, seconds, threads):
    """Oracle throughput (Mcell-layer-steps/s) over about `seconds` of work."""
    import oracle
    gomp = ctypes.CDLL("libgomp.so.1")
    oracle.lib()
    gomp.omp_set_num_threads(int(threads))
    o = oracle.Oracle(b)
    o.set_state(p, p)
    o.set_forcing(w, None, ts, tn)
    o.step(tdt, 1)                      # warm-up (FFT plans, first touch)
    n, t0 = 0, time.perf_counter()
    while True:
        o.step(tdt, 1)
        n += 1
        el = time.perf_counter() - t0
        if el >= seconds and n >= 2:
            break
    o.close()
    cells = b.nxp * b.nyp * b.nl
    return cells * n / el / 1e6, n, el


def dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def run_reference(args):
    """The reference arm: the CPU restatement of step_qg (the oracle, FP64,
    OpenMP on the leapfrog region only, as the reference parallelises it)
    on the host cores local to the GPU.  It is timed with one thread and
    with every bound thread; the faster is the line's value, with its thread
    count (the reference's only parallel region is a small share of the
    step, so more threads can be slower)."""
    ws, rank, local = dist()
    if rank != 0:
        return 0
    numa_cpus = None
    try:
        import torch
        if torch.cuda.is_available():
            numa_cpus = bind_to_gpu_numa(local)
    except Exception:
        pass
    from openqg_b200.params import OQG_FP64
    b, tdt, label = make_basin(args.workload, OQG_FP64)
    p, w, ts, tn = initial_inputs(b, seed=1, reference=True)
    import oracle
    gomp = ctypes.CDLL("libgomp.so.1")
    oracle.lib()
    allt = len(os.sched_getaffinity(0)) or (os.cpu_count() or 1)
    msteps = args.ref_model_steps
    cells = b.nxp * b.nyp * b.nl
    runs = {}
    for threads in sorted({1, allt}):
        gomp.omp_set_num_threads(threads)
        o = oracle.Oracle(b)
        o.set_state(p, p)
        o.set_forcing(w, None, ts, tn)
        for _ in range(args.warmup):
            o.step(tdt, msteps)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            o.step(tdt, msteps)
        el = time.perf_counter() - t0
        o.close()
        runs[threads] = (cells * msteps * args.steps / el / 1e6, el)
    threads = max(runs, key=lambda t: runs[t][0])
    value, el = runs[threads]
    line = {
        "impl": "reference", "metric": "Mcell-layer-steps/s", "value": value,
        "unit": "Mcell-layer-steps/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": el * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": label, "nxp": b.nxp, "nyp": b.nyp, "nl": b.nl,
                   "model_steps_per_step": msteps, "tdt_s": tdt, "parallelism": "single process"},
        "cpu_baseline": {"value": value, "unit": "Mcell-layer-steps/s", "cores": threads,
                         "kind": "port",
                         "sample": "%d x %d model steps of the %s basin (FP64 C++ restatement of the "
                                   "Fortran step_qg, OpenMP on the leapfrog region only), the faster of "
                                   "1 and %d threads" % (args.steps, msteps, args.workload, allt),
                         "by_threads": {str(t): v[0] for t, v in sorted(runs.items())},
                         "host_cpus_bound": numa_cpus},
        "e2e": {"value": value, "unit": "Mcell-layer-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def bind_to_gpu_numa(device_index):
    """Pins this process to the host CPUs local to the GPU (from sysfs), so
    pinned host buffers and the copy engines sit on the same NUMA node.
    Returns the CPU count bound to, or None when the topology is unknown."""
    import torch
    try:
        pr = torch.cuda.get_device_properties(device_index)
        bus = "%04x:%02x:%02x.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
        with open("/sys/bus/pci/devices/%s/local_cpulist" % bus) as f:
            spec = f.read().strip()
        cpus = set()
        for part in spec.split(","):
            if "-" in part:
                a, b = part.split("-")
                cpus.update(range(int(a), int(b) + 1))
            elif part:
                cpus.add(int(part))
        cpus &= os.sched_getaffinity(0)
        if cpus:
            os.sched_setaffinity(0, cpus)
            return len(cpus)
    except Exception:
        pass
    return None


def max_over_ranks(ms, pg, device):
    """Max of a per-rank time over all ranks; every rank calls it."""
    import torch
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    if pg is not None:
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def replica_value(total_ms, ws, cells, msteps, steps):
    """Whole-job Mcell-layer-steps/s of ws replicas that each ran the same work."""
    return ws * cells * msteps * steps / (total_ms / 1e3) / 1e6


def time_batches(g, tdt, msteps, steps, flush):
    import torch
    s = torch.cuda.ExternalStream(g.stream())
    total = 0.0
    # an NVTX range marks the timed steps for a profiler's filter
    torch.cuda.nvtx.range_push("timed_steps")
    for _ in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        g.step(tdt, msteps)
        e1.record(s)
        e1.synchronize()
        total += e0.elapsed_time(e1)
    torch.cuda.nvtx.range_pop()
    g.sync()
    return total


PHASES = ["k_vort", "k_xfwd", "k_ysolve", "k_xinv"]
# a closed box runs the inverse transforms and the assembly as two launches
PHASES_SEP = ["k_vort", "k_xfwd", "k_ysolve", "k_xinv_rows", "k_xinv_asm"]


def phase_alg_bytes(s, nl):
    """Algorithmic bytes per cell-layer of each step phase (s: bytes per
    state word)."""
    return {
        # reads p, q, pm, qm (+ wekp once per column of layers); writes q, modal rhs
        "k_vort": 6 * s + s / nl,
        # reads the modal rhs, writes its transform
        "k_xfwd": 2 * s,
        # reads and writes the spectral field (+ FP64 pivots, not counted)
        "k_ysolve": 2 * s,
        # reads the spectral field, p (old) and the homogeneous solutions, writes p
        "k_xinv": 3 * s + s * (nl - 1) / nl,
        # reads the spectral field, writes the modal rows
        "k_xinv_rows": 2 * s,
        # reads the modal rows and the homogeneous solutions, writes p
        "k_xinv_asm": 2 * s + s * (nl - 1) / nl,
    }


def roofline_of(g, b, workload, precision, tdt, ms_per_model_step):
    """The dominant phase timed alone (oqg_profile_phases: CUDA events around
    each kernel of 20 steps) against the HBM roofline, and the whole step's
    algorithmic bytes over its timed duration."""
    from openqg_b200.params import OQG_FP64
    names = PHASES_SEP if g.xinv_sep() else PHASES
    ms = g.profile_phases(tdt, 20)[:len(names)]
    dom = int(np.argmax(ms))
    s = 8 if b.precision == OQG_FP64 else 4
    cells = b.nxp * b.nyp * b.nl
    alg = phase_alg_bytes(s, b.nl)
    peak, peak_kind = peaks()
    dname = names[dom]
    achieved = alg[dname] * cells / (ms[dom] / 1e3) / 1e9
    step_alg = (6 * s + s / b.nl) * cells
    tt = traffic_table().get((workload, precision, dname))
    return {"bound": "hbm", "kernel": dname, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_kind": peak_kind,
            "traffic": tt, "alg_bytes_per_launch": alg[dname] * cells,
            "phase_ms": dict(zip(names, [float(x) for x in ms])),
            "step_alg_bytes": step_alg,
            # the whole step: algorithmic bytes over the timed model step
            "step_frac": step_alg / (ms_per_model_step / 1e3) / 1e9 / peak,
            # the phases timed one by one, summed
            "phases_frac": step_alg / (sum(ms) / 1e3) / 1e9 / peak,
            # the step chain's launches with no work (oqg_launch_floor): the
            # most a single persistent launch could take off a step
            "launch_floor_us_per_step": g.launch_floor(16),
            "launches_per_step": g.step_launches()}


# --tile-rows / --ysolve-warps: settings fixed instead of measured (for
# profiling runs, where a profiler's replays would distort the measurement)
PINNED = {}


def measure_basin(workload, prec, steps, warmup, msteps, flush, rank, pg, seed=None):
    """Device throughput of one basin: autotuned tiles, `warmup` untimed
    batches, then `steps` batches of msteps model steps, each after an L2
    flush; the time is the max over ranks.  Returns the handle (open), the
    basin, its inputs and the figures."""
    from openqg_b200.core import QG
    b, tdt, label = make_basin(workload, prec)
    p, w, ts, tn = initial_inputs(b, seed=(1 + rank) if seed is None else seed)
    g = QG(b)
    g.set_state(p, p)
    g.set_forcing(w, None, ts, tn)
    # the vorticity tile height and the y-solve's warps per column, measured
    # on this GPU (oqg_autotune, oqg_autotune_ysolve), unless fixed
    if PINNED.get("tile_rows"):
        g.set_tile_rows(PINNED["tile_rows"])
        tile_rows, tune_ms = PINNED["tile_rows"], {}
    else:
        tile_rows, tune_ms = g.autotune(tdt, 20)
    if PINNED.get("xinv_sep") is not None:
        g.set_xinv_sep(PINNED["xinv_sep"])
        xsep, xtune_ms = bool(PINNED["xinv_sep"]), {}
    else:
        xsep, xtune_ms = g.autotune_xinv(tdt, 20)
    if PINNED.get("ysolve_warps"):
        g.set_ysolve_warps(PINNED["ysolve_warps"])
        ywarps, ytune_ms = PINNED["ysolve_warps"], {}
    else:
        ywarps, ytune_ms = g.autotune_ysolve(tdt, 20)
    for _ in range(warmup):
        g.step(tdt, msteps)
    g.sync()
    if g.check_finite() != 0:
        raise RuntimeError("non-finite state after warm-up (%s)" % workload)
    if pg:
        pg.barrier()
    total_ms = max_over_ranks(time_batches(g, tdt, msteps, steps, flush), pg, "cuda")
    cells = b.nxp * b.nyp * b.nl
    return g, b, (p, w, ts, tn), {
        "workload": label, "tdt_s": tdt, "label": label, "total_ms": total_ms,
        "ms_per_model_step": total_ms / (steps * msteps), "cells": cells,
        "tile_rows": tile_rows, "autotune_ms_per_step": {str(k): round(v, 5) for k, v in tune_ms.items()},
        "ysolve_warps": ywarps, "ysolve_autotune_ms_per_step": {str(k): round(v, 5) for k, v in ytune_ms.items()},
        "xinv_two_launches": xsep,
        "xinv_autotune_ms_per_step": {("two launches" if k else "one kernel"): round(v, 5)
                                      for k, v in xtune_ms.items()},
    }


def config_line(workload, prec, steps, warmup, msteps, flush, rank, ws, pg, note=""):
    """A whole-configuration figure with its own roofline (a variant of the
    bench line)."""
    from openqg_b200.params import OQG_FP64
    g, b, _, m = measure_basin(workload, prec, steps, warmup, msteps, flush, rank, pg)
    pname = "fp64" if prec == OQG_FP64 else "mixed"
    roof = roofline_of(g, b, workload, pname, m["tdt_s"], m["ms_per_model_step"])
    g.close()
    return {"workload": m["label"] + note, "precision": pname, "tdt_s": m["tdt_s"],
            "model_steps_per_step": msteps, "steps": steps,
            "value": replica_value(m["total_ms"], ws, m["cells"], msteps, steps),
            "unit": "Mcell-layer-steps/s", "ms_per_model_step": m["ms_per_model_step"],
            "tile_rows": m["tile_rows"], "ysolve_warps": m["ysolve_warps"],
            "xinv_two_launches": m["xinv_two_launches"], "roofline": roof,
            "l2": "flushed (256 MiB write) before every timed step of %d model steps" % msteps}


def e2e_breakdown(g, b, L, wk_p, ent_p, p1_p, ts, tn, tdt, reps=20):
    """Host-clock medians of the three parts of an exchanged model step:
    the forcing upload (oqg_set_forcing, which returns once the copies have
    read the host arrays), the step alone, and the read-back of p(:,:,1)."""
    def med(fn):
        ts_ = []
        for _ in range(reps):
            g.sync()
            t0 = time.perf_counter()
            fn()
            g.sync()
            ts_.append((time.perf_counter() - t0) * 1e3)
        return statistics.median(ts_)
    up = med(lambda: L.oqg_set_forcing(g.h, wk_p, ent_p, ts, tn))
    st = med(lambda: L.oqg_step(g.h, tdt, 1))
    rd = med(lambda: L.oqg_get_p_layer(g.h, 0, p1_p))
    return {"upload_ms": up, "step_ms": st, "readback_ms": rd}


def run_ours(args):
    import torch
    ws, rank, local = dist()
    torch.cuda.set_device(local)
    numa_cpus = bind_to_gpu_numa(local)
    pg = None
    if ws > 1:
        import datetime
        import torch.distributed as td
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                              device_id=torch.device("cuda", local))
        pg = td
    from openqg_b200.core import lib
    from openqg_b200.params import OQG_FP64, OQG_MIXED
    prec = OQG_MIXED if args.precision == "mixed" else OQG_FP64
    msteps = args.model_steps
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")   # 256 MiB > L2

    def barrier():
        if pg:
            pg.barrier()
        torch.cuda.synchronize()

    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(local).uuid)
    except Exception:
        pass
    barrier()
    with Clocks(uuid) as clk:
        g, b, (p, w, ts, tn), m = measure_basin(args.workload, prec, args.steps, args.warmup, msteps, flush,
                                                rank, pg)
        barrier()
    tdt, label, cells = m["tdt_s"], m["label"], m["cells"]
    total_ms = m["total_ms"]
    value = replica_value(total_ms, ws, cells, msteps, args.steps)

    # e2e through the C ABI with pinned host buffers
    L = lib()
    wk_h = torch.empty(b.shape2, dtype=torch.float64, pin_memory=True)
    wk_h.copy_(torch.from_numpy(w))
    ent_h = torch.zeros((b.nl - 1,) + b.shape2, dtype=torch.float64, pin_memory=True)
    p1_h = torch.empty(b.shape2, dtype=torch.float64, pin_memory=True)
    dp = ctypes.POINTER(ctypes.c_double)
    wk_p = ctypes.cast(wk_h.data_ptr(), dp)
    ent_p = ctypes.cast(ent_h.data_ptr(), dp)
    p1_p = ctypes.cast(p1_h.data_ptr(), dp)
    e2e_steps = max(1, min(args.steps, 10))

    def exchange_step():
        for _ in range(msteps):
            rc = L.oqg_set_forcing(g.h, wk_p, ent_p, ts, tn)
            rc |= L.oqg_step(g.h, tdt, 1)
            rc |= L.oqg_get_p_layer(g.h, 0, p1_p)
            if rc:
                raise RuntimeError(L.oqg_last_error().decode())

    exchange_step()
    barrier()
    # each bench step is timed on the host clock (every call returns only
    # after its copies completed); the median step time is reported, so one
    # step stalled by other host activity does not set the figure
    e2e_times = []
    for _ in range(e2e_steps):
        t0 = time.perf_counter()
        exchange_step()
        g.sync()
        e2e_times.append((time.perf_counter() - t0) * 1e3)
    e2e_ms = max_over_ranks(statistics.median(e2e_times) * e2e_steps, pg, "cuda")
    e2e_value = replica_value(e2e_ms, ws, cells, msteps, e2e_steps)
    e2e_parts = e2e_breakdown(g, b, L, wk_p, ent_p, p1_p, ts, tn, tdt)
    # wekp + the ent layers the step reads (a box: ent(:,:,1); a channel: all nl-1)
    h2d = msteps * (b.nxp * b.nyp * 8) * (b.nl if b.cyclic else 2)
    d2h = msteps * b.nxp * b.nyp * 8
    coupled = None
    if prec == OQG_FP64 and not b.cyclic:
        coupled = coupled_e2e(g, b, tdt, msteps, e2e_steps)

    # the dominant kernel, timed alone, against the HBM roofline
    g.set_forcing(w, None, ts, tn)
    roof = roofline_of(g, b, args.workload, args.precision, tdt, m["ms_per_model_step"])

    variants = {}
    if args.variants and prec == OQG_FP64:
        # the same basin with FP32 bulk arithmetic
        variants["mixed_fp32_bulk"] = config_line(args.workload, OQG_MIXED, args.steps, args.warmup, msteps,
                                                  flush, rank, ws, pg)
        # the plain configuration: 129x129x3, dx 20 km, 480 leapfrog steps
        # (one bench step is the whole run)
        variants["config0_ocean129_480steps"] = config_line("ocean129", OQG_FP64, 3, args.warmup, 480, flush,
                                                            rank, ws, pg)
        # the eddy-resolving box, FP64 and FP32 bulk
        for vprec, vname in ((OQG_FP64, "ocean2049_fp64"), (OQG_MIXED, "ocean2049_mixed")):
            variants[vname] = config_line("ocean2049", vprec, max(3, args.steps // 2), args.warmup, msteps,
                                          flush, rank, ws, pg)
        # the batched ensemble: 256 basins of uneven size, one launch per phase;
        # with N ranks each steps every N-th member (no collective), so the
        # whole ensemble is stepped once per step across the ranks
        for vprec, vname in ((OQG_MIXED, "ensemble256_mixed"), (OQG_FP64, "ensemble256_fp64")):
            cells_e, te, rows_e = run_ensemble(vprec, args.steps, args.warmup, msteps, flush, rank=rank, ws=ws)
            te = max_over_ranks(te, pg, "cuda")
            variants[vname] = replica_value(te, 1, cells_e, msteps, args.steps)
            variants[vname + "_tile_rows"] = rows_e
        variants["ensemble_config"] = ("256 ocean 3-layer boxes, sizes uniform in %s, dx 20 km, "
                                       "per-member wind 0.05-0.15 N/m^2 and ah4 1e10-4e10; %d "
                                       "cell-layers per step, sharded by member over %d rank(s) "
                                       "(strong scaling, no collective)" % (list(ENSEMBLE_SIZES), cells_e, ws))
        # the coupled configuration's step loop with both mixed layers on the device
        variants["coupled_config"] = coupled_config()
        variants["coupled_config_fp32_bulk"] = coupled_config(precision=OQG_MIXED)
        # the adjoint: reverse pass and adjoint step against the forward step
        variants["adjoint257"] = run_adjoint()
        # the eddy-resolving box: forward + adjoint over 100 steps, checkpoint every 10
        adx, aah4, atdt = ADJOINT_BOXES[2049]
        variants["adjoint2049"] = run_adjoint(reps=1, n=2049, dx=adx, ah4=aah4, nsteps=100, every=10, tdt=atdt)

    line = {
        "metric": "Mcell-layer-steps/s", "value": value, "unit": "Mcell-layer-steps/s",
        "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if prec == OQG_FP64 else "f32+f64",
        "data": "synthetic",
        "config": {"workload": label, "nxp": b.nxp, "nyp": b.nyp, "nl": b.nl,
                   "model_steps_per_step": msteps, "tdt_s": tdt,
                   "tile_rows": m["tile_rows"],
                   "autotune_ms_per_step": m["autotune_ms_per_step"],
                   "ysolve_warps": m["ysolve_warps"],
                   "ysolve_autotune_ms_per_step": m["ysolve_autotune_ms_per_step"],
                   "xinv_two_launches": m["xinv_two_launches"],
                   "xinv_autotune_ms_per_step": m["xinv_autotune_ms_per_step"],
                   "l2": "flushed (256 MiB write) before every timed step of %d model steps" % msteps,
                   "parallelism": "replicas" if ws > 1 else "single basin"},
        "roofline": roof,
        "e2e": {"value": e2e_value, "unit": "Mcell-layer-steps/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "timer": "host clock, median of %d steps" % e2e_steps,
                "pattern": "per model step: upload wekp+ent (the layers the step reads), step, read p(:,:,1)",
                "parts_ms_per_model_step": e2e_parts},
        "e2e_coupled_ocean": coupled,
        "gpu_launches": args.steps * msteps * launches_per_step(g),
        "host_cpus_bound": numa_cpus,
        "clocks": clk.summary(),
        "variants": variants,
    }
    if rank == 0 and ws == 1 and args.cpu_seconds > 0:
        from openqg_b200.params import OQG_FP64 as F64
        b64, _, _ = make_basin(args.workload, F64)
        v, n, el = cpu_sample(b64, p, w, ts, tn, tdt, args.cpu_seconds, 1)
        line["cpu_baseline"] = {"value": v, "unit": "Mcell-layer-steps/s", "cores": 1, "kind": "port",
                                "sample": "%d model steps of the same basin in %.1f s (FP64 C++ restatement "
                                          "of the Fortran step_qg, 1 thread)" % (n, el)}
    g.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


def launches_per_step(g):
    """Kernel launches of one model step of the handle's step path."""
    return g.step_launches()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="ocean513", choices=sorted(WORKLOADS))
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--model-steps", type=int, default=10)
    ap.add_argument("--ref-model-steps", type=int, default=2)
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-variants", dest="variants", action="store_false")
    ap.add_argument("--tile-rows", type=int, default=0, choices=[0, 8, 12, 16],
                    help="fix the vorticity tile height instead of measuring it")
    ap.add_argument("--xinv-sep", type=int, default=None, choices=[0, 1],
                    help="the inverse transforms as a launch of their own (1) or inside the assembly "
                         "kernel (0); default: measured")
    ap.add_argument("--ysolve-warps", type=int, default=0, choices=[0, 1, 2, 4],
                    help="fix the y-solve's warps per column instead of measuring them")
    ap.add_argument("--adjoint-only", action="store_true",
                    help="time only the adjoint configuration (one repetition of 40 steps) and "
                         "print its figures; for profiling")
    ap.add_argument("--adjoint-n", type=int, default=257, choices=sorted(ADJOINT_BOXES),
                    help="box size of --adjoint-only")
    ap.add_argument("--ensemble-only", action="store_true",
                    help="time only the 256-member ensemble (--precision) and print its figure; for profiling")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    PINNED["tile_rows"] = args.tile_rows
    PINNED["ysolve_warps"] = args.ysolve_warps
    PINNED["xinv_sep"] = args.xinv_sep
    if args.impl == "reference":
        return run_reference(args)
    if args.adjoint_only:
        import torch
        torch.cuda.set_device(0)
        dx, ah4, tdt = ADJOINT_BOXES[args.adjoint_n]
        print(json.dumps(run_adjoint(reps=1, n=args.adjoint_n, dx=dx, ah4=ah4, nsteps=40, every=20, tdt=tdt)),
              flush=True)
        return 0
    if args.ensemble_only:
        import torch
        from openqg_b200.params import OQG_FP64, OQG_MIXED
        torch.cuda.set_device(0)
        flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
        prec = OQG_MIXED if args.precision == "mixed" else OQG_FP64
        cells, te, rows = run_ensemble(prec, args.steps, args.warmup, args.model_steps, flush)
        print(json.dumps({"ensemble256": args.precision, "value": replica_value(te, 1, cells, args.model_steps, args.steps),
                          "unit": "Mcell-layer-steps/s", "tile_rows": rows}), flush=True)
        return 0
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
