"""Benchmark: DOF-updates/s of the RK4 DG shallow-water step (SPOC cal_var path).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl spoc|reference]
                  [--config c2_fs_p6]

Workload: configuration C2 of the reference's benchmark set (nonlinear
free-slip calvarnl_fs, degree 6 = 28 modes, tri2_33 / legen7 quadrature,
2 x 128 x 128 = 32768 jittered triangles on a 1000 km beta-plane basin,
8 seeded geostrophic Gaussians), synthetic and seeded.  A step is one
classical RK4 step (4 right-hand sides + update).  Metric:
DOF-updates/s = 3 * nm * ne * steps / seconds (u, v, eta), whole job.

`value`: device-resident state, CUDA events around every step on the
launching stream, L2 flushed (256 MiB write) before every timed step, max
over ranks.  `e2e`: the host-buffer entry point spoc_rk4_steps_host, one step
per call with pinned host arrays, inside the timed region: the state copied
host->device, the step, and the new state stored back into the pinned arrays
by the last stage kernel (mapped host memory) as it computes it.  N > 1 runs independent replicas (one per GPU, no
collective on the data path): weak scaling.

--impl reference times the CPU restatement of the reference (oracle/,
OpenMP over all host cores) on the same workload: rank 0 only.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "DOF-updates/s per RK4 step (plain FP64 vs mixed/adjoint) at stated L2 error"
UNIT = "DOF-updates/s"


def workload_desc(cfg, ne, nm):
    return (f"{cfg.name}: cal_var {cfg.variant} degree {cfg.nc} (nm={nm}), tri2_{cfg.ng}/legen{cfg.ngf}, "
            f"2x{cfg.n}x{cfg.n}={ne} triangles (jitter {cfg.jitter}), {cfg.length / 1e3:.0f} km basin, "
            f"f0={cfg.f0}, beta={cfg.beta}, mu0={cfg.mu0}, mb0={cfg.mb0}, H={cfg.depth}, ic={cfg.ic}")


PRECISION_DESC = {
    "fp64": "fp64, reference operation order (GPU bit-exact to the CPU oracle)",
    "fp64_fma": "fp64 with fused multiply-adds (not bit-exact)",
    "mixed": "FP32 contractions in the orthonormal basis, FP64 RK4 state",
}


def workload_config(cfg, ne, nm, dt, precision, n_gpus):
    """The `config` object of both arms (identical on both for the same
    workload, precision and GPU count)."""
    return {"workload": workload_desc(cfg, ne, nm), "ne": ne, "nm": nm, "dt": dt,
            "precision": PRECISION_DESC[precision],
            "l2": "GPU arm: L2 flushed (256 MiB write) before every timed step; "
                  "CPU arm: no flush (the state, 22 MB per field at C2, streams from DRAM)",
            "parallelism": (f"replicas x{n_gpus} (GPU arm); CPU arm on rank 0's host cores"
                            if n_gpus > 1 else
                            "single device (GPU arm: one GPU; CPU arm: OpenMP over the host cores)")}


def model_counts_mixed(cfg, ne):
    """Per-kernel algorithmic FP32 flops and compulsory HBM bytes of one
    mixed-precision RHS (kx_vol, kx_tend; kx_lin for the linear variant).

    Flops: the multiply-adds the kernels issue (2 flops each).  Bytes: own
    element reads and writes (state FP32 / FP64, partial load vectors, trace
    records of 3*ngf + 1 floats; a neighbour's record counted once more).
    """
    N, Q, G = cfg.nm, cfg.ng, cfg.ngf
    TG, TS = 3 * G, 3 * G + 1
    rk4_bytes = 3 * N * (8 + 8 + 8 + 4)  # c64 read, acc read+write, y write
    if cfg.variant == "lin":
        macs = 6 * N * (N - 1) + 3 * TG * N + 3 * TG * (N - 1)
        return {"kx_lin": (2.0 * ne * macs, ne * (3 * N * 4 + 2 * 3 * TS * 4 + rk4_bytes + 3 * TS * 4))}
    vol = 4 * N * (N - 1) + 4 * TG * N + 3 * Q * N + 4 * Q * N + 4 * Q * N + 6 * N * (N - 1) + 6 * TG * (N - 1)
    tend = 3 * TG * N + 3 * TG * (N - 1)
    return {
        "kx_vol": (2.0 * ne * vol, ne * (3 * N * 4 + 2 * 2 * TS * 4 + 2 * Q * 4 + 3 * N * 4 + 6 * TS * 4)),
        "kx_tend": (2.0 * ne * tend, ne * (3 * N * 4 + 2 * 7 * TS * 4 + rk4_bytes + 3 * TS * 4)),
    }


def mnorm_factory(p):
    det = p.mesh.det
    A = p.T.ammo.T

    def mnorm(x):
        return float(np.sqrt(np.sum(det * np.einsum("ei,ij,ej->e", x, A, x))))
    return mnorm


def timed_steps(torch, stream, flush, s, dt, nsteps):
    """ms per RK4 step over nsteps single-step calls, L2 flushed before each."""
    out = []
    for _ in range(nsteps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            flush.zero_()
            a.record(stream)
        s.rk4_steps(dt, 1)
        with torch.cuda.stream(stream):
            b.record(stream)
        b.synchronize()
        out.append(a.elapsed_time(b))
    return sum(out) / nsteps


def timed_call(torch, stream, flush, s, dt, nsteps, repeats=3):
    """ms per RK4 step of one rk4_steps(dt, nsteps) call (L2 flushed before
    the call), the median of `repeats` calls."""
    out = []
    for _ in range(repeats):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            flush.zero_()
            a.record(stream)
        s.rk4_steps(dt, nsteps)
        with torch.cuda.stream(stream):
            b.record(stream)
        b.synchronize()
        out.append(a.elapsed_time(b) / nsteps)
    return sorted(out)[len(out) // 2]


def mixed_measure(torch, stream, flush, W, api, name="c3_inv_p7", steps=1000, tsteps=10):
    """Mixed-precision form against plain FP64 on one configuration, with the
    volume work on the FP32 pipes (the default) and on the tensor cores: ms
    per step, relative L2 errors of u, v, eta after `steps` steps, energy
    drift of every run, and the roofline of the dominant mixed kernel."""
    cfg = W.CONFIGS[name]
    p = W.build_problem(cfg)
    mnorm = mnorm_factory(p)
    dof = 3.0 * p.T.nm * p.mesh.ne
    runs = [("fp64", "fp64", "auto"), ("mixed", "mixed", "templated"), ("mixed_tensor", "mixed", "tensor")]
    res, states, drift, kms = {}, {}, {}, {}
    for key, prec, path in runs:
        s = W.make_solver(p, prec)
        s.set_kernel_path(path)
        s.set_stream(stream.cuda_stream)
        s.set_state(p.u, p.v, p.h)
        s.rk4_steps(p.dt, 3)
        res[key] = timed_steps(torch, stream, flush, s, p.dt, tsteps)
        s.set_state(p.u, p.v, p.h)
        e0 = s.energy()
        s.rk4_steps(p.dt, steps)
        e1 = s.energy()
        states[key] = s.get_state()
        drift[key] = ((e1[0] + e1[1]) - (e0[0] + e0[1])) / (e0[0] + e0[1])
        if prec == "mixed":
            s.set_state(p.u, p.v, p.h)
            kms[key] = s.profile_rk4(p.dt, 2)
        s.close()

    def errs(key):
        return {f: mnorm(states[key][i] - states["fp64"][i]) / mnorm(states["fp64"][i])
                for i, f in enumerate(("u", "v", "eta"))}

    counts = model_counts_mixed(cfg, p.mesh.ne)
    per_launch = {n: float(kms["mixed"][i]) / 8 for i, n in enumerate(counts)}
    tcounts = {("kt_vol" if k == "kx_vol" else k): v for k, v in counts.items()}
    per_launch_tc = {n: float(kms["mixed_tensor"][i]) / 8 for i, n in enumerate(tcounts)}
    dom = max(per_launch, key=per_launch.get)
    fl, by = counts[dom]
    dur = per_launch[dom] * 1e-3
    fp32 = api.fp64_peak(2)
    return {
        "config": f"{name}: {p.mesh.ne} triangles, degree {cfg.nc} (nm={p.T.nm}), dt={p.dt}",
        "fp64_ms_per_step": res["fp64"], "mixed_ms_per_step": res["mixed"],
        "fp64_value": dof / (res["fp64"] * 1e-3), "mixed_value": dof / (res["mixed"] * 1e-3),
        "speedup": res["fp64"] / res["mixed"],
        "steps_compared": steps, "rel_l2_error_vs_fp64": errs("mixed"),
        "energy_drift": {"fp64": drift["fp64"], "mixed": drift["mixed"]},
        "energy_drift_difference": drift["mixed"] - drift["fp64"],
        "kernel_ms_per_launch": per_launch,
        "roofline": {"kernel": dom, "bound": "fp32", "achieved": fl / dur / 1e12, "peak": fp32,
                     "unit": "TFLOP/s", "frac": fl / dur / 1e12 / fp32,
                     "hbm_gbs": by / dur / 1e9, "traffic": ncu_traffic(name, dom)[0],
                     "traffic_note": ncu_traffic(name, dom)[1],
                     "peak_source": "measured live: spoc_fp64_peak mode 2 (FP32 FMA chains)"},
        "tensor_core_path": {
            "volume_kernel": "kt_vol: tcgen05 TF32 MMAs (3-term split), accumulators in TMEM",
            "ms_per_step": res["mixed_tensor"], "value": dof / (res["mixed_tensor"] * 1e-3),
            "speedup": res["fp64"] / res["mixed_tensor"],
            "rel_l2_error_vs_fp64": errs("mixed_tensor"),
            "energy_drift": drift["mixed_tensor"],
            "kernel_ms_per_launch": per_launch_tc,
            "traffic_kt_vol": ncu_traffic(name, "kt_vol")[0]},
    }


def fp64_configs_measure(torch, stream, flush, W, names=("c1_lin_p3", "c4_ns_p4"), steps=20,
                         call_steps=100):
    """Plain FP64 step of the other single-GPU configurations (C3 in
    mixed_measure), DOF-updates/s from ms per RK4 step of one
    rk4_steps(dt, call_steps) call (L2 flushed before the call: how a run of
    many steps is made); beside it the ms per step of single-step calls (L2
    flushed before each; host launch cost and the per-call flag read
    included)."""
    out = {}
    for name in names:
        p = W.build_problem(W.CONFIGS[name])
        s = W.make_solver(p)
        s.set_stream(stream.cuda_stream)
        s.set_state(p.u, p.v, p.h)
        s.rk4_steps(p.dt, 3)
        l0 = s.launches
        ms1 = timed_steps(torch, stream, flush, s, p.dt, steps)
        per1 = (s.launches - l0) / steps
        l0 = s.launches
        ms = timed_call(torch, stream, flush, s, p.dt, call_steps)
        dof = 3.0 * p.T.nm * p.mesh.ne
        out[name] = {"ne": p.mesh.ne, "nm": p.T.nm, "ms_per_step": ms,
                     "value": dof / (ms * 1e-3), "unit": UNIT,
                     "steps_per_call": call_steps,
                     "launches_per_call": (s.launches - l0) / 3,
                     "ms_per_step_single_step_calls": ms1,
                     "launches_per_single_step_call": per1}
        s.close()
        # the mixed-precision form on the same workload, timed the same way
        m = W.make_solver(p, "mixed")
        m.set_stream(stream.cuda_stream)
        m.set_state(p.u, p.v, p.h)
        m.rk4_steps(p.dt, 3)
        mms = timed_call(torch, stream, flush, m, p.dt, call_steps)
        out[name].update({"mixed_ms_per_step": mms, "mixed_value": dof / (mms * 1e-3),
                          "mixed_speedup": ms / mms})
        m.close()
    return out


MIXED_RUNS = {"c1_lin_p3": 1000, "c2_fs_p6": 2000, "c4_ns_p4": 200}


def mixed_errors_all(W):
    """Mixed-precision form against FP64 on C1, C2 and C4 at their full sizes
    and run lengths (C3 in mixed_measure, C5 in ensemble_measure): relative L2
    errors of u, v, eta and both runs' energy drift."""
    out = {}
    for name, steps in MIXED_RUNS.items():
        p = W.build_problem(W.CONFIGS[name])
        out[name] = W.precision_errors(p, steps)
    return out


def ensemble_measure(torch, stream, W, api, replicas, rank=0, world=1, count=64, steps=500):
    """Configuration C5: 64 free-slip members of degree 3-6 on their own
    refined meshes (4k-40k triangles), mixed precision, stepped together (one
    cooperative launch per RK4 stage, CUDA graph); the layout is picked by
    the autotuner.  Reports the aggregate DOF-updates/s over `steps` steps and
    each member's relative L2 eta error against its own FP64 run."""
    t0 = time.perf_counter()
    allm = W.ensemble_members(count, seed=5)
    ps = [W.build_member(allm[i]) for i in replicas.member_share(count, rank, world)]
    build_s = time.perf_counter() - t0
    dts = [p.dt for p in ps]
    mem = []
    for p in ps:
        s = W.make_solver(p, "mixed")
        s.set_state(p.u, p.v, p.h)
        mem.append(s)
    ens = api.Ensemble(mem)
    tune = ens.autotune(dts, 3)
    for p, s in zip(ps, mem):
        s.set_state(p.u, p.v, p.h)
    ens.steps(dts, 2)  # graph capture and warm-up
    for p, s in zip(ps, mem):
        s.set_state(p.u, p.v, p.h)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    ens.steps(dts, steps)
    b.record()
    b.synchronize()
    ms = a.elapsed_time(b)
    info = ens.info()
    dof = sum(3.0 * p.T.nm * p.mesh.ne for p in ps)
    # members split across GPUs (replicas): all ranks' work over the slowest time
    ms_all, units = replicas.reduce_throughput(ms, dof * steps, world, "cuda")
    errs, uv_errs, drifts = [], [], []
    for p, s in zip(ps, mem):
        ref = W.run_steps(p, "fp64", steps)
        mn = mnorm_factory(p)
        got = s.get_state()
        e = [mn(got[i] - ref[0][i]) / mn(ref[0][i]) for i in range(3)]
        errs.append(e[2])
        uv_errs.append(max(e[0], e[1]))
        e_end = s.energy()
        drifts.append((W.energy_drift(ref[1], ref[2]), W.energy_drift(ref[1], e_end)))
    ens.close()
    for s in mem:
        s.close()
    if world > 1:
        import torch.distributed as dist
        gathered = [None] * world
        dist.all_gather_object(gathered, (errs, uv_errs, drifts))
        errs = [e for g in gathered for e in g[0]]
        uv_errs = [e for g in gathered for e in g[1]]
        drifts = [e for g in gathered for e in g[2]]
    ddiff = [abs(m - f) for f, m in drifts]
    ne = np.array([p.mesh.ne for p in ps])
    mb = np.array(info["member_blocks"])
    return {
        "config": f"c5: {count} calvarnl_fs members, degree 3-6, refined meshes, own dt each, "
                  f"{steps} steps; this rank: {len(ps)} members, {int(ne.min())}-{int(ne.max())} "
                  f"triangles ({int(ne.sum())} in all)",
        "value": units / (ms_all * 1e-3), "unit": UNIT, "ms_per_step": ms_all / steps,
        "dof_per_step": units / steps, "members_split_over_ranks": world,
        "precision": "mixed (FP32 contractions, FP64 state)",
        "launches_per_step": 4, "graph": info["graph"],
        "autotuner": {"best": tune["best"], "tried": tune["tried"],
                      "blocks": info["blocks"],
                      "elements_per_block": {"min": float((ne / mb).min()), "max": float((ne / mb).max())},
                      "warps_per_block": 8,
                      "elements_per_warp": {"degree 3-4": 2, "degree 5-6": 1}},
        "eta_rel_l2_error_vs_fp64": {"max": float(max(errs)), "median": float(np.median(errs)),
                                     "members": [float(e) for e in errs]},
        "uv_rel_l2_error_vs_fp64": {"max": float(max(uv_errs)),
                                    "median": float(np.median(uv_errs))},
        "energy_drift": {"fp64_median": float(np.median([f for f, _ in drifts])),
                         "mixed_median": float(np.median([m for _, m in drifts])),
                         "max_abs_difference": float(max(ddiff))},
        "host_setup_s": build_s,
    }


def host_rk4_step(rhs, u0, v0, h0, dt, w):
    """One RK4 step driven the way the reference's loop drives cal_var
    (src/shwwnl.f:233-284): four right-hand sides on host arrays, the stage
    states and the final combination computed on the host in the same
    operation order (numpy, in place; w holds the work arrays)."""
    x0 = (u0, v0, h0)
    d = w["d"]
    y = w["y"]
    t = w["t"]
    for k in range(4):
        rhs(*(x0 if k == 0 else y), *d[k])
        if k < 3:
            for f in range(3):
                np.multiply(d[k][f], dt, out=t)
                if k < 2:
                    np.multiply(t, 0.5, out=t)
                np.add(x0[f], t, out=y[f])
    dt6 = dt / 6.0
    for f in range(3):
        np.multiply(d[1][f], 2.0, out=t)
        np.add(d[0][f], t, out=t)
        np.multiply(d[2][f], 2.0, out=y[f])
        np.add(t, y[f], out=t)
        np.add(t, d[3][f], out=t)
        np.multiply(t, dt6, out=t)
        np.add(x0[f], t, out=x0[f])


def drop_in_measure(torch, W, api, p, steps=5):
    """The literal drop-in, driven as the Fortran driver drives it: every RK4
    step makes four cal_var calls on host arrays and does the stage AXPYs on
    the host.  Two entries: cal_var_ (the reference's 31 by-reference
    arguments, arrays with the reference's leading dimension nnmod = 45,
    pageable memory) and the handle entry spoc_cal_var (packed ld = nm arrays
    in pinned memory).  Host wall clock, synchronous calls; the final state
    is checked bit for bit against the device-resident run."""
    import ctypes as C
    cfg, m = p.cfg, p.mesh
    ne, nm, ld = m.ne, p.T.nm, 45
    dof = 3.0 * nm * ne

    def pad(a):
        out = np.zeros((ne, ld))
        out[:, :nm] = a[:, :nm]
        return out

    # reference: the device-resident path from the same state
    s = W.make_solver(p)
    s.set_state(p.u, p.v, p.h)
    s.rk4_steps(p.dt, steps + 1)
    ref = s.get_state()
    s.close()
    res = {}
    # ---- cal_var_ (31 by-reference arguments), ld = 45, pageable ----
    lib = api.load_library()
    T45 = p.T
    # the COMMON matrices with the reference's leading dimension nnmod = 45,
    # which is also the leading dimension cal_var_ takes for the state arrays
    mats = {}
    for name in ("amm", "amml", "agx", "agy", "ammo"):
        a = np.zeros((nm, ld))
        a[:, :nm] = getattr(T45, name)
        mats[name] = a
    ts = api._Tables(T45.nc, nm, T45.ng, T45.ngf, api._d(T45.wi), api._d(T45.xi), api._d(T45.yi),
                     api._d(T45.wif), api._d(T45.tif), api._d(T45.pi2), T45.ng, api._d(T45.pico),
                     T45.ngf, nm, api._d(mats["amm"]), api._d(mats["amml"]), api._d(mats["agx"]),
                     api._d(mats["agy"]), api._d(mats["ammo"]), ld, api._i(T45.cip))
    assert lib.spoc_register_commons(C.byref(ts), api.VARIANTS[cfg.variant], api.FP64) == 0
    keep = []

    def ints(x):
        keep.append(C.c_int(x))
        return C.c_void_p(C.addressof(keep[-1]))

    def dbl(x):
        keep.append(C.c_double(x))
        return C.c_void_p(C.addressof(keep[-1]))

    ptr = lambda a: C.c_void_p(a.ctypes.data)
    fc, w0, z0, hb = (pad(a) for a in (p.fc, p.w0, p.z0, p.hb))
    pbdl = np.zeros(ne, np.int32)
    pint = np.zeros(ne, np.int32)
    fixed = dict(tseg=ptr(m.tseg), pseg=ptr(m.pseg), ssit=ptr(m.ssit), itm=ptr(m.itm),
                 its=ptr(m.its), norm=ptr(m.norm), bdl=ptr(m.bdl), cip=ptr(T45.cip),
                 vect=ptr(m.vect), normt=ptr(m.normt))

    def cal_var_(u0, v0, h0, u1, v1, h1):
        lib.cal_var_(ints(m.nf), ints(ne), ptr(u0), ptr(v0), ptr(h0), ptr(u1), ptr(v1), ptr(h1),
                     fixed["tseg"], fixed["pseg"], fixed["ssit"], fixed["itm"], fixed["its"],
                     fixed["norm"], ints(0), ptr(pbdl), ints(0), ptr(pint), fixed["bdl"],
                     fixed["cip"], fixed["vect"], fixed["normt"], dbl(cfg.mu0), dbl(cfg.mb0),
                     ptr(fc), dbl(cfg.beta), ptr(w0), ptr(z0), dbl(cfg.g0), ptr(hb), dbl(0.0))
        del keep[:]
        if lib.spoc_cal_var_status()[0] != 0:
            raise RuntimeError("cal_var_ failed: " + str(lib.spoc_last_error()))

    in_calls = [0.0]

    def run(rhs, alloc):
        x = [alloc(a) for a in (p.u, p.v, p.h)]
        w = {"d": [[alloc(None) for _ in range(3)] for _ in range(4)],
             "y": [alloc(None) for _ in range(3)], "t": alloc(None)}

        def timed_rhs(*args):
            t = time.perf_counter()
            rhs(*args)
            in_calls[0] += time.perf_counter() - t

        host_rk4_step(rhs, *x, p.dt, w)  # warm-up (upload of the mesh on the first call)
        torch.cuda.synchronize()
        in_calls[0] = 0.0
        t0 = time.perf_counter()
        for _ in range(steps):
            host_rk4_step(timed_rhs, *x, p.dt, w)
        sec = time.perf_counter() - t0
        same = all(np.array_equal(x[i][:, :nm], ref[i][:, :nm]) for i in range(3))
        return sec, same

    sec, same = run(cal_var_, lambda a: pad(a) if a is not None else np.zeros((ne, ld)))
    lib.spoc_release_commons()
    res["cal_var_"] = {
        "value": dof * steps / sec, "unit": UNIT, "ms_per_step": 1e3 * sec / steps,
        "ms_per_call": 1e3 * in_calls[0] / (4 * steps),
        "host_axpy_ms_per_step": 1e3 * (sec - in_calls[0]) / steps,
        "h2d_bytes_per_step": 4 * 3 * ne * nm * 8, "d2h_bytes_per_step": 4 * 3 * ne * nm * 8,
        "arrays": "pageable numpy, leading dimension 45 (nnmod)",
        "bitwise_equal_to_device_resident_run": same}
    # ---- spoc_cal_var (handle), ld = nm, pinned ----
    s = W.make_solver(p)

    def pinned(a):
        t = torch.zeros((ne, nm), dtype=torch.float64).pin_memory()
        if a is not None:
            t.numpy()[...] = a[:, :nm]
        keep_pin.append(t)
        return t.numpy()

    keep_pin = []

    def handle_rhs(u0, v0, h0, u1, v1, h1):
        api._check(api.load_library().spoc_cal_var(s._h, nm, api._d(u0), api._d(v0), api._d(h0),
                                                   api._d(u1), api._d(v1), api._d(h1)),
                   "cal_var")

    sec, same = run(handle_rhs, pinned)
    s.close()
    res["spoc_cal_var"] = {
        "value": dof * steps / sec, "unit": UNIT, "ms_per_step": 1e3 * sec / steps,
        "ms_per_call": 1e3 * in_calls[0] / (4 * steps),
        "host_axpy_ms_per_step": 1e3 * (sec - in_calls[0]) / steps,
        "h2d_bytes_per_step": 4 * 3 * ne * nm * 8, "d2h_bytes_per_step": 4 * 3 * ne * nm * 8,
        "arrays": "pinned, packed (ld = nm)",
        "bitwise_equal_to_device_resident_run": same}
    res["note"] = ("4 cal_var calls per RK4 step on host arrays, stage AXPYs on the host "
                   f"(numpy); host wall clock over {steps} steps after one warm-up step")
    return res


def model_counts(cfg, ne, nf):
    """Per-kernel algorithmic FP64 flops and compulsory HBM bytes of one RHS.

    Flops count the reference's multiply-adds (2 flops each): cal_b N^2,
    DTRSM4 N^2 per solve (two half sweeps), spectoxy/xytospec Q*N, tri_f 3*N*G,
    cal_flu 2*N*G per face (both sides).  Bytes: each kernel's own-element
    reads and writes of modal fields (neighbour data is an L2 re-read).
    """
    N, Q, G = cfg.nm, cfg.ng, cfg.ngf
    if cfg.variant == "lin":
        macs = ne * (6 * N * N + 3 * N * N + 4 * 3 * N * G) + nf * 3 * 2 * N * G
        return {"kf_lin": (2.0 * macs, 8.0 * ne * N * (3 + 9))}
    return {
        "kf_qphase": (2.0 * (ne * (8 * N * N + 12 * N * G) + nf * 2 * 2 * N * G), 8.0 * ne * N * (2 + 4)),
        "kf_nlvol": (2.0 * ne * (2 * N * N + 17 * Q * N), 8.0 * ne * N * (11 + 8)),
        "kf_tend": (2.0 * (ne * (15 * N * N + 18 * N * G) + nf * 6 * 2 * N * G), 8.0 * ne * N * (8 + 12)),
    }


# DRAM bytes (read + write) per launch of a kernel on a workload, each from one
# ncu capture of that kernel, with the SHA-256 prefix of the kernel's source
# file at the capture: a figure is reported only while the source is unchanged
# (otherwise `traffic` is null, since it would describe another version).
KERNEL_SOURCE = {"kf_": "spoc_fast.cu", "kx_": "spoc_mixed.cu", "kt_": "spoc_mixed_tc.cu"}
# At C2 the q-phase and tendency phases are two launches each (the face values
# once per face, kf_faces, then kf_qphasef / kf_tendf): their figures are the
# sums over the phase's two kernels.
NCU_TRAFFIC = {
    "c2_fs_p6:kf_qphase": (39800320, "3d82445bfb57b56a"),
    "c2_fs_p6:kf_nlvol": (98205184, "3d82445bfb57b56a"),
    "c2_fs_p6:kf_tend": (167291904, "3d82445bfb57b56a"),
    "c3_inv_p7:kx_vol": (248066048, "6bbf3e429a3ee218"),
    "c3_inv_p7:kx_tend": (578007040, "6bbf3e429a3ee218"),
}
# The kernels behind each timed phase of the FP64 nonlinear RHS at the
# degrees whose modes fit one row per lane (3-6).
PHASE_KERNELS = {"kf_qphase": "kf_faces<NF=2> (face values of u, v) + kf_qphasef",
                 "kf_nlvol": "kf_nlvol",
                 "kf_tend": "kf_faces<NF=6> (face values of f, uh, vh) + kf_tendf"}


def source_digest(kernel: str):
    for prefix, fname in KERNEL_SOURCE.items():
        if kernel.startswith(prefix):
            data = (ROOT / "spoc_b200" / "csrc" / fname).read_bytes()
            return hashlib.sha256(data).hexdigest()[:16]
    return None


def ncu_traffic(config: str, kernel: str):
    """(bytes per launch, note): the ncu figure if it was captured on this
    version of the kernel's source, else (None, why)."""
    ent = NCU_TRAFFIC.get(f"{config}:{kernel}")
    if ent is None:
        return None, "no ncu capture of this kernel on this workload"
    nbytes, digest = ent
    now = source_digest(kernel)
    if digest is None or digest != now:
        return None, f"ncu capture predates the current kernel source ({now})"
    return nbytes, f"ncu dram__bytes_read.sum + dram__bytes_write.sum, kernel source {now}"


def sample_clocks_start(out: Path):
    q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    try:
        f = open(out, "w")
        return subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                 "-lms", "200"], stdout=f, stderr=subprocess.DEVNULL), f
    except Exception:
        return None, None


def sample_clocks_stop(proc, fh, out: Path, gpu_index: int):
    if proc is None:
        return None
    proc.terminate()
    try:
        proc.wait(timeout=5)
    except Exception:
        proc.kill()
    fh.close()
    sm, mx, reasons = [], None, set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for line in out.read_text().splitlines():
        parts = [p.strip() for p in line.split(",")]
        if len(parts) < 9 or not parts[0].isdigit() or int(parts[0]) != gpu_index:
            continue
        try:
            sm.append(float(parts[1]))
            mx = float(parts[2])
        except ValueError:
            continue
        for name, val in zip(names, parts[5:9]):
            if val.lower().startswith("active"):
                reasons.add(name)
    if not sm:
        return None
    return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
            "samples": len(sm)}


def run_reference(args, cfg, rank):
    """CPU restatement of the reference (oracle/), all host threads, rank 0
    only.  The workload is set up by the oracle itself (oracle.problems): the
    CUDA library is not loaded by this arm."""
    if rank != 0:
        return
    from oracle import oracle as O
    from oracle.problems import oracle_problem

    P = oracle_problem(cfg)
    threads = O.default_threads()
    u, v, h = P.u.copy(), P.v.copy(), P.h.copy()

    def step():
        P.rk4(u, v, h, 1, threads)

    nwarm = max(1, args.warmup)
    t0 = time.perf_counter()
    for _ in range(nwarm):
        step()
    per = (time.perf_counter() - t0) / nwarm
    budget = 120.0
    k = max(1, min(args.steps, int(budget / max(per, 1e-9))))
    t0 = time.perf_counter()
    for _ in range(k):
        step()
    sec = time.perf_counter() - t0
    ne, nm = P.M.ne, P.T.nm
    dof = 3.0 * nm * ne
    val = dof * k / sec
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus,
        "steps": k, "warmup": nwarm, "ms_per_step": 1e3 * sec / k, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(cfg, ne, nm, P.dt, "fp64", args.gpus),
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{k} full RK4 steps of the workload ({args.steps} requested, "
                                   f"capped at {budget:.0f} s)"},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def cpu_baseline(cfg):
    """Oracle on the host cores, bounded to ~10-30 s (rank 0, N=1), on the
    oracle's own set-up of the workload."""
    from oracle import oracle as O
    from oracle.problems import oracle_problem
    P = oracle_problem(cfg)
    threads = O.default_threads()
    dof = 3.0 * P.T.nm * P.M.ne
    u, v, h = P.u.copy(), P.v.copy(), P.h.copy()
    k, t0 = 0, time.perf_counter()
    while True:
        P.rk4(u, v, h, 1, threads)
        k += 1
        sec = time.perf_counter() - t0
        if sec > 10.0 or k >= 50:
            break
    # the serial reference: one core, at least one step, about 6 s
    u, v, h = P.u.copy(), P.v.copy(), P.h.copy()
    k1, t0 = 0, time.perf_counter()
    while True:
        P.rk4(u, v, h, 1, 1)
        k1 += 1
        sec1 = time.perf_counter() - t0
        if sec1 > 6.0 or k1 >= 20:
            break
    return {"value": dof * k / sec, "unit": UNIT, "cores": threads,
            "kind": "port", "sample": f"{k} full RK4 steps of the workload, OpenMP over elements",
            "serial": {"value": dof * k1 / sec1, "unit": UNIT, "cores": 1,
                       "sample": f"{k1} full RK4 steps of the workload on one core"}}


def adjoint_measure(torch, stream, nsteps=200, snaps=20, nobs=500):
    """Configuration C4: gradient of the observation cost over a 200-step
    window of calvarnl_ns (p4, 32768 triangles) with 20 binomial snapshots;
    500 seeded points observed at steps 50/100/150/200 against a truth run."""
    from spoc_b200 import workloads as W
    cfg = W.CONFIGS["c4_ns_p4"]
    p = W.build_problem(cfg)
    s = W.make_solver(p)
    s.set_stream(stream.cuda_stream)
    W.assimilation_window(p, s, nobs, steps=(50, 100, 150, 200))
    x0 = (p.u, p.v, p.h)
    s.fwd_window(x0, p.dt, nsteps)  # warm-up

    def timed(fn):
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        out = fn()
        b.record(stream)
        b.synchronize()
        return out, a.elapsed_time(b)

    # median of three runs of each window
    fw = [timed(lambda: s.fwd_window(x0, p.dt, nsteps)) for _ in range(3)]
    J, t_fwd = fw[0][0], float(np.median([t for _, t in fw]))
    s.adjoint_counters()
    bw = [timed(lambda: s.bwd_window(x0, p.dt, nsteps, snaps)) for _ in range(3)]
    (J2, g), t_bwd = bw[0][0], float(np.median([t for _, t in bw]))
    nf, na = s.adjoint_counters()
    nf, na = nf // 3, na // 3
    # the forward sweeps in the mixed-precision form (adjoint kernels FP64)
    s.set_adjoint_sweeps("mixed")
    bm = [timed(lambda: s.bwd_window(x0, p.dt, nsteps, snaps)) for _ in range(3)]
    (Jm, gm), t_bm = bm[0][0], float(np.median([t for _, t in bm]))
    s.set_adjoint_sweeps("fp64")
    g_rel = (sum(float(np.sum((a - b) ** 2)) for a, b in zip(gm, g)) /
             sum(float(np.sum(b * b)) for b in g)) ** 0.5
    s.close()
    # the mixed-precision forward over the same window (the RK4 steps alone,
    # one call, median of three)
    m = W.make_solver(p, "mixed")
    m.set_stream(stream.cuda_stream)
    m.set_state(*x0)
    m.rk4_steps(p.dt, nsteps)
    t_mix = []
    for _ in range(3):
        m.set_state(*x0)
        t_mix.append(timed(lambda: m.rk4_steps(p.dt, nsteps))[1])
    t_mix = float(np.median(t_mix))
    m.close()
    return {"config": f"c4_ns_p4: {p.mesh.ne} triangles, nm={p.T.nm}, window {nsteps} steps, "
                      f"{snaps} binomial snapshots, {nobs} observation points at steps 50/100/150/200",
            "cost": J, "forward_window_ms": t_fwd, "gradient_ms": t_bwd,
            "timing": "median of three runs of each window",
            "gradient_over_forward": t_bwd / t_fwd,
            "mixed_forward_window_ms": t_mix,
            "gradient_over_mixed_forward": t_bwd / t_mix,
            "gradient_precision": "fp64 (the gradient of the FP64 forward; no mixed-precision "
                                  "tangent-linear or adjoint kernels)",
            "mixed_sweeps": {
                "what": "spoc_set_adjoint_sweeps(SPOC_MIXED): the cost sweep, the checkpoint "
                        "sweeps and the re-advances in the mixed-precision form; tangent-linear "
                        "and adjoint kernels FP64, linearised about that trajectory",
                "gradient_ms": t_bm, "gradient_over_forward": t_bm / t_fwd,
                "gradient_over_mixed_forward": t_bm / t_mix,
                "gradient_rel_l2_difference_vs_fp64": g_rel,
                "cost_rel_difference_vs_fp64": abs(Jm - J2) / abs(J2)},
            "forward_steps_run_by_gradient": nf, "adjoint_steps": na,
            "checks": "dot-product, central differences (20 directions) and checkpointing invariance in tests/test_gpu_adjoint.py"}


def regrid_measure(torch, stream, fp64_mul_add, name="c2_fs_p6", steps=20, reps=10):
    """Solution-driven regridding of the C2 state after `steps` RK4 steps: the
    error indicator (cal_conv), refinement of the elements above the 90th
    percentile of the indicator, the host point location, the device
    re-projection (interpol) of u, v, eta, verif_rot and checkcfl2.  Kernel
    times by CUDA events on the handles' stream; the oracle's interpol (one
    core, walk included) is timed beside it on the same meshes."""
    from spoc_b200 import api
    from spoc_b200 import workloads as W
    cfg = W.CONFIGS[name]
    p = W.build_problem(cfg)
    s = W.make_solver(p)
    s.set_stream(stream.cuda_stream)
    s.set_state(p.u, p.v, p.h)
    s.rk4_steps(p.dt, steps)

    def timed(fn, n=reps):
        out, ms = None, []
        for _ in range(n):
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            out = fn()
            b.record(stream)
            b.synchronize()
            ms.append(a.elapsed_time(b))
        return out, float(np.median(ms))

    amax = np.maximum.reduce(s.checkconv())
    fac1 = float(np.quantile(amax, 0.9))
    cc, t_conv = timed(lambda: s.cal_conv(fac1, 0.0, 10.0 * fac1))
    t0 = time.perf_counter()
    p1, tinter, loc = W.adapt_problem(p, cc["fconv"])
    t_adapt = time.perf_counter() - t0
    t0 = time.perf_counter()
    api.locate_points(p.mesh, p1.mesh, tinter, p.T)
    t_walk = time.perf_counter() - t0
    d = api.Solver(p1.T, p1.mesh, cfg.variant)
    d.set_params(cfg.mu0, cfg.mb0, cfg.g0, p1.hb, p1.fc, p1.w0, p1.z0)
    d.set_stream(stream.cuda_stream)
    dev = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (tinter, *loc)]
    ptrs = [t.data_ptr() for t in dev]
    l0 = d.launches
    d.interpol_from_dev(s, *ptrs)
    _, t_interp = timed(lambda: d.interpol_from_dev(s, *ptrs))
    launches = (d.launches - l0) / (reps + 1)
    t0 = time.perf_counter()
    for _ in range(3):
        d.interpol_from(s, tinter, *loc)
    t_e2e = (time.perf_counter() - t0) / 3 * 1e3
    _, t_rot = timed(d.verif_rot)
    (cflmin, dt2), t_cfl2 = timed(lambda: d.cfl2(10, p.dt))
    nm, ng, ne1 = p.T.nm, p.T.ng, p1.mesh.ne
    nproj = int((tinter == 0).sum())
    flops = nproj * (2 * 9.0 * nm * ng + 6.0 * nm * nm)
    byts = nproj * (ng * 20.0 + 2 * 3 * nm * 8) + (ne1 - nproj) * 2 * 3 * nm * 8
    # CPU baseline: the oracle's interpol (walk included), one core, same meshes
    from oracle import oracle as O
    T = p.T
    OT = O.Tables(cfg.nc, cfg.ng, cfg.ngf, T.wi, T.xi, T.yi, T.wif, T.tif)
    OM = O.Mesh(p.mesh.inn, p.mesh.xgr, p.mesh.ygr, cfg.nc, cfg.f0, cfg.beta)
    NM = O.Mesh(p1.mesh.inn, p1.mesh.xgr, p1.mesh.ygr, cfg.nc, cfg.f0, cfg.beta)
    u, v, h = s.get_state()
    t0 = time.perf_counter()
    for a in (u, v, h):
        O.interpol(OT, OM, NM, tinter, a)
    t_cpu = time.perf_counter() - t0
    dof = 3.0 * nm * ne1
    s.close()
    d.close()
    return {
        "config": f"{name}: {p.mesh.ne} -> {ne1} triangles after {steps} RK4 steps; elements with "
                  f"an indicator above its 90th percentile refined (red + green closure); "
                  f"{nproj} re-projected, {ne1 - nproj} inherited",
        "metric": "re-projected DOF per second (interpol of u, v, eta)",
        "value": dof / (t_interp * 1e-3), "unit": "DOF/s",
        "interpol_ms": t_interp, "interpol_launches_per_call": launches,
        "e2e": {"value": dof / (t_e2e * 1e-3), "unit": "DOF/s", "ms": t_e2e,
                "note": "spoc_interpol with host arrays (point tables uploaded inside)"},
        "cal_conv_ms": t_conv, "verif_rot_ms": t_rot, "cfl2_ms": t_cfl2,
        "cfl2": {"cflmin": cflmin, "dt": dt2},
        "host_refine_s": t_adapt, "host_walk_s": t_walk,
        "roofline": {"kernel": "k_interpol", "bound": "fp64",
                     "achieved": flops / (t_interp * 1e-3) / 1e12, "peak": fp64_mul_add,
                     "unit": "TFLOP/s", "frac": flops / (t_interp * 1e-3) / 1e12 / fp64_mul_add,
                     "algorithmic_flops_per_call": flops, "algorithmic_bytes_per_call": byts,
                     "hbm_gbs": byts / (t_interp * 1e-3) / 1e9,
                     "peak_source": "measured live: spoc_fp64_peak mode 1 (separate DMUL + DADD)"},
        "cpu_baseline": {"value": dof / t_cpu, "unit": "DOF/s", "cores": 1, "kind": "port",
                         "sample": "the oracle's interpol of u, v, eta on the same meshes, walk included"},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="spoc", choices=["spoc", "reference"])
    ap.add_argument("--config", default="c2_fs_p6")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--no-regrid", action="store_true")
    ap.add_argument("--no-drop-in", action="store_true")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp64_fma", "mixed"],
                    help="fp64: bit-exact reference order (headline); fp64_fma: fused "
                         "multiply-adds; mixed: FP32 contractions, FP64 state")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    from spoc_b200 import workloads as W
    cfg = W.CONFIGS[args.config]

    if args.impl == "reference":
        run_reference(args, cfg, rank)
        return

    import torch
    import torch.distributed as dist
    from spoc_b200 import api, replicas

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    p = W.build_problem(cfg)
    ne, nm = p.mesh.ne, p.T.nm
    s = W.make_solver(p, args.precision)
    stream = torch.cuda.Stream()
    s.set_stream(stream.cuda_stream)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    s.set_state(p.u, p.v, p.h)
    s.rk4_steps(p.dt, args.warmup)

    # ---- timed region: device-resident state ----
    clk_dir = tempfile.TemporaryDirectory(prefix="spoc_bench_clocks_")
    clk_file = Path(clk_dir.name) / f"clocks_rank{rank}.csv"
    proc, fh = sample_clocks_start(clk_file) if rank == 0 else (None, None)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = s.launches
    times = []
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    for i in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
            ev[i][0].record(stream)
        s.rk4_steps(p.dt, 1)
        with torch.cuda.stream(stream):
            ev[i][1].record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    launches = s.launches - l0
    clocks = sample_clocks_stop(proc, fh, clk_file, local) if rank == 0 else None
    times = [a.elapsed_time(b) for a, b in ev]
    total_ms = float(sum(times))
    dof = 3.0 * nm * ne
    # replicas: all ranks' work over the slowest rank's time
    total_ms, units = replicas.reduce_throughput(total_ms, dof * args.steps, world, "cuda")
    value = units / (total_ms * 1e-3)

    # ---- e2e: host buffers through spoc_rk4_steps_host ----
    pin = [torch.from_numpy(a.copy()).pin_memory() for a in (p.u, p.v, p.h)]
    host = [t.numpy() for t in pin]
    e2e_steps = max(3, min(args.steps, 10))
    s.rk4_steps_host(*host, p.dt, 1)  # warm-up
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e_times = []
    for _ in range(e2e_steps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        s.rk4_steps_host(*host, p.dt, 1)
        b.record(stream)
        b.synchronize()
        e_times.append(a.elapsed_time(b))
    e_ms, e_units = replicas.reduce_throughput(float(sum(e_times)), dof * e2e_steps, world, "cuda")
    e2e = {"value": e_units / (e_ms * 1e-3), "unit": UNIT,
           "h2d_bytes_per_step": 3 * ne * nm * 8, "d2h_bytes_per_step": 3 * ne * nm * 8}

    # ---- e2e through the literal drop-in: 4 cal_var calls per step ----
    drop_in = None
    if world == 1 and not args.no_drop_in and args.precision == "fp64":
        drop_in = drop_in_measure(torch, W, api, p)

    # ---- per-kernel timing and roofline of the dominant kernel ----
    s.set_state(p.u, p.v, p.h)
    prof_steps = 2
    kms = s.profile_rk4(p.dt, prof_steps)
    counts = model_counts(cfg, ne, p.mesh.nf) if args.precision != "mixed" else model_counts_mixed(cfg, ne)
    names = list(counts)
    per_launch_ms = {n: float(kms[i]) / (4 * prof_steps) for i, n in enumerate(names)}
    dom = max(per_launch_ms, key=per_launch_ms.get)
    fl, by = counts[dom]
    dur = per_launch_ms[dom] * 1e-3
    fp64_fma = api.fp64_peak(0)
    fp64_mul_add = api.fp64_peak(1)
    try:
        hbm_peak = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())["hbm_gbs"]
        hbm_src = "measured (MEASURED_PEAKS.json hbm_gbs)"
    except Exception:
        hbm_peak, hbm_src = 6650.0, "fallback (6.65 TB/s, earlier measurement on this GPU type)"
    traffic, traffic_note = ncu_traffic(cfg.name, dom)
    hbm = {"achieved": by / dur / 1e9, "peak": hbm_peak, "unit": "GB/s",
           "frac": by / dur / 1e9 / hbm_peak, "algorithmic_bytes_per_launch": by,
           "peak_source": hbm_src}
    # the binding resource: the FP64 (or, mixed, FP32) pipe of the dominant
    # kernel, against the measured peak of the arithmetic the kernel must use
    if args.precision == "mixed":
        fp32 = api.fp64_peak(2)
        roof = {"kernel": dom, "bound": "fp32", "achieved": fl / dur / 1e12, "peak": fp32,
                "unit": "TFLOP/s", "frac": fl / dur / 1e12 / fp32, "traffic": traffic,
                "traffic_note": traffic_note, "algorithmic_flops_per_launch": fl,
                "launch_ms": per_launch_ms[dom],
                "peak_source": "measured live: spoc_fp64_peak mode 2 (FP32 FMA chains)",
                "hbm": hbm}
    else:
        pk = fp64_mul_add if args.precision == "fp64" else fp64_fma
        roof = {"kernel": dom, "bound": "fp64", "achieved": fl / dur / 1e12, "peak": pk,
                "unit": "TFLOP/s", "frac": fl / dur / 1e12 / pk, "traffic": traffic,
                "traffic_note": traffic_note, "algorithmic_flops_per_launch": fl,
                "launch_ms": per_launch_ms[dom],
                "peak_source": ("measured live: spoc_fp64_peak mode 1, separately rounded DMUL + "
                                "DADD (the arithmetic the bit-exact path must use), 2 flops per pair"
                                if args.precision == "fp64" else
                                "measured live: spoc_fp64_peak mode 0, DFMA chains"),
                "frac_of_dfma_peak": fl / dur / 1e12 / fp64_fma, "dfma_peak": fp64_fma,
                "hbm": hbm}

    # the other precision modes on the same workload, and their distance from
    # the headline run after 100 steps
    mnorm = mnorm_factory(p)
    s.set_state(p.u, p.v, p.h)
    s.rk4_steps(p.dt, 100)
    ref_state = s.get_state()
    others = []
    for other in [x for x in ("fp64", "fp64_fma", "mixed") if x != args.precision]:
        s2 = W.make_solver(p, other)
        s2.set_stream(stream.cuda_stream)
        s2.set_state(p.u, p.v, p.h)
        s2.rk4_steps(p.dt, args.warmup)
        ms = timed_steps(torch, stream, flush, s2, p.dt, args.steps)
        s2.set_state(p.u, p.v, p.h)
        s2.rk4_steps(p.dt, 100)
        st2 = s2.get_state()
        s2.close()
        others.append({"precision": other, "value": dof / (ms * 1e-3), "ms_per_step": ms,
                       "rel_l2_diff_after_100_steps": {
                           f: mnorm(st2[i] - ref_state[i]) / mnorm(ref_state[i])
                           for i, f in enumerate(("u", "v", "eta"))}})

    fp64_configs = None
    if world == 1 and args.precision == "fp64":
        fp64_configs = fp64_configs_measure(torch, stream, flush, W)
    mixed = mixed_all = None
    if world == 1 and not args.no_mixed:
        mixed = mixed_measure(torch, stream, flush, W, api)
        mixed_all = mixed_errors_all(W)
    ensemble = None
    if not args.no_ensemble:
        ensemble = ensemble_measure(torch, stream, W, api, replicas, rank, world)

    adjoint = None
    if world == 1 and not args.no_adjoint:
        adjoint = adjoint_measure(torch, stream)
    regrid = None
    if world == 1 and not args.no_regrid:
        regrid = regrid_measure(torch, stream, fp64_mul_add)

    line = None
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision != "mixed" else "f32 contractions / f64 state",
            "data": "synthetic",
            "config": workload_config(cfg, ne, nm, p.dt, args.precision, world),
            "e2e": e2e,
            "e2e_drop_in": drop_in,
            "gpu_launches": int(launches),
            "kernel_ms_per_launch": per_launch_ms,
            "phase_kernels": (PHASE_KERNELS if args.precision == "fp64" and cfg.variant != "lin"
                              and nm <= 32 else None),
            "roofline": roof,
            "other_precisions": others,
            "fp64_other_configs": fp64_configs,
            "mixed_c3": mixed,
            "mixed_errors": mixed_all,
            "ensemble_c5": ensemble,
            "adjoint": adjoint,
            "regrid": regrid,
            "clocks": clocks,
        }
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(cfg)
        print(json.dumps(line), flush=True)
    s.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
