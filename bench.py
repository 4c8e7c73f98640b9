"""RI J+K Fock-build throughput on one B200 (and N replicas under torchrun).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (the synthetic nonrelativistic RI J/K kernel configuration): n = 400 AOs, naux = 1600,
nocc = 40; AO and aux centres uniform in a 20-bohr cube, B^P_mn = c_Pmn exp(-0.3(|r_m-r_P|^2 +
|r_n-r_P|^2)) with c symmetric N(0,1); D = 2 C_occ C_occ^T with C_occ a QR-orthonormalised
Gaussian 400 x 40; S = X = I.  One step = one full FP64 RI Fock build F = h + J - K/2 through
rr_ri_fock_nonrel (occupied recovery, J, K, assembly) -- the reference's nonRelFockMatrix.
B is 2.05 GB, far larger than the 126 MB L2, so no flush is needed between steps.

Multi-GPU: the path is replicas only (each rank builds its own Fock matrices on its own
copy of B; no collective), value = total builds/s over all ranks, timed as the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

N_AO, N_AUX, N_OCC, SEED = 400, 1600, 40, 2024
# The half-transform kernel of the nonrelativistic exchange (RR_HALF_TRANSFORM selects it; m16 is the
# library default) with the DRAM bytes (read + write) of one launch at this workload from its ncu
# capture (B read once, T written once), None where no capture exists.
HT_KIND = os.environ.get("RR_HALF_TRANSFORM", "m16").split(":")[0]
HT_KERNELS = {
    "m8": dict(kernel="dgemm_kernel half-transform T^P = Ct B^P (FP64 DMMA m8n8k4)",
               traffic=2.048888e9 + 0.194917e9, profile="profiles/dgemm_half_transform_n400_naux1600_nocc40.md"),
    "m16": dict(kernel="ht_dmma16_kernel half-transform T^P = Ct B^P (FP64 DMMA m16n8k8)",
                traffic=2.048169e9 + 0.197358e9,
                profile="profiles/ht_dmma16_half_transform_n400_naux1600_nocc40.md"),
}
HT = HT_KERNELS[HT_KIND]
METRIC = "RI J+K Fock builds/s"
UNIT = "builds/s"


def bench_config(world_size: int) -> dict:
    """The workload description both arms print (the GPU arm and --impl reference)."""
    return {"workload": f"nonrel RI J+K Fock build n={N_AO} naux={N_AUX} nocc={N_OCC} (FP64, occupied recovery "
                        f"included)", "parallelism": f"replicas x{world_size}", "precision": "fp64",
            "l2": "inputs larger than L2 (B = 2.05 GB)"}


def cpu_model() -> str:
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def make_inputs():
    from rerdmft_b200 import synth

    rng = np.random.default_rng(SEED + 1)
    B = synth.ri_tensor(N_AO, N_AUX, SEED, box=20.0, alpha=0.3)
    C, D = synth.occupied_density(N_AO, N_OCC, rng)
    a = rng.standard_normal((N_AO, N_AO))
    h = 0.5 * (a + a.T)
    return dict(B=B, C=C, D=D, h=h, S=np.eye(N_AO), X=np.eye(N_AO))


def make_scf_system():
    """SCF inputs of the same shape (n=400, naux=1600, nocc=40): rerdmft_b200.synth.nonrel_system with a
    0.5 Ha core gap and the two-electron part scaled by 8 (B by sqrt 8) so that the orbitals change
    over the iterations (the reference's loop needs 9 of them), an overlap near identity, its
    canonical X and the core-guess density."""
    from rerdmft_b200 import synth

    s = synth.nonrel_system(N_AO, N_AUX, N_OCC, seed=SEED + 7, box=20.0, gap=0.5)
    s["B"] *= np.sqrt(8.0)
    return s


NL4, NS4, NAUX4, NOCC4 = 200, 600, 1000, 40


def rkb_fock_times(torch, fp64_peak, want_cpu: bool, steps: int = 10):
    """4-component Kramers-restricted RKB Fock build (rkbFockMatrix) at nl=200, ns=600, naux=1000,
    20 Kramers pairs: LL and SS tensors by the cube/Gaussian recipe (20-bohr cube), device-resident,
    timed with CUDA events; the reference's own rkbFockMatrix timed once on the host cores."""
    import ctypes

    from rerdmft_b200 import _lib as L
    from rerdmft_b200 import ri, synth

    s = synth.rkb_system(NL4, NS4, NAUX4, 2 * (NOCC4 // 2), seed=SEED + 11, box=20.0)
    dev = {k: torch.from_numpy(np.ascontiguousarray(s[k])).cuda()
           for k in ("B_LL", "B_SS", "v_total", "s_full", "x_full", "h", "P0")}
    src = ri.RiDirectEriSource(NL4, NS4, dev["B_LL"], dev["B_SS"], dev["v_total"], dev["s_full"], dev["x_full"])
    store = src.store
    lib = L.lib()
    n_rkb = s["n_rkb"]
    F = torch.empty((n_rkb, n_rkb), dtype=torch.complex128, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    o = L.opts(L.RR_MEM_DEVICE, stream=stream, sync=0)
    x = dev["x_full"]

    def step():
        L.check(lib.rr_ri_fock_rkb(store.handle, dev["h"].data_ptr(), dev["v_total"].data_ptr(), n_rkb,
                                   dev["s_full"].data_ptr(), x.data_ptr(), x.shape[1], dev["P0"].data_ptr(),
                                   F.data_ptr(), ctypes.byref(o)))

    for _ in range(3):
        step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    store.sync()
    ms = e0.elapsed_time(e1) / steps
    fl = [NL4, NL4, NS4, NS4]
    pair = sum(fl[f] * fl[u] for f in range(4) for u in range(f, 4))
    flops = 4.0 * NOCC4 * (2 * NL4 ** 2 + 2 * NS4 ** 2) * NAUX4 + 8.0 * NOCC4 * pair * NAUX4
    tf = flops / (ms / 1e3) / 1e12
    out = dict(workload=f"rkbFockMatrix nl={NL4} ns={NS4} naux={NAUX4} nocc={NOCC4} spinors (FP64 complex)",
               ms_per_build=ms, builds_per_s=1e3 / ms, algorithmic_gflop=flops / 1e9, achieved_tflops=tf,
               frac_of_dgemm=(tf / fp64_peak) if fp64_peak else None,
               j_bytes=2.0 * NAUX4 * (NL4 ** 2 + NS4 ** 2) * 8)
    if want_cpu:
        from oracle import ref

        if ref.available():
            ref.set_threads(os.cpu_count() or 1)
            t0 = time.perf_counter()
            F_ref = ref.rkb_fock(s["h"], NL4, NS4, s["B_LL"], s["B_SS"], s["v_total"], s["s_full"], s["x_full"],
                                 s["P0"])
            dt = time.perf_counter() - t0
            out["reference_cpu"] = dict(seconds_per_build=dt, cores=os.cpu_count() or 1, cpu_model=cpu_model(),
                                        sample="one full-size call of the reference rkbFockMatrix")
            out["parity"] = dict(max_abs_F_minus_reference=float(np.abs(F.cpu().numpy() - F_ref).max()),
                                 tolerance=1e-10, inputs="the timed build's inputs")
    del dev, src, store, F
    torch.cuda.empty_cache()
    return out


def mo_transform_block(torch, fp64_peak, want_cpu: bool, reps: int = 5):
    """MO three-index transforms of the functional stage: buildRiNonRelSpinMoEri at the headline shape
    (n = 400, naux = 1600, C a full 400 x 400 orthogonal matrix: 4 naux n^3 = 409.6 GFLOP) and buildRiMoEri
    at the 4-component shapes (nl = 200, ns = 600, naux = 1000, 400 positive-energy spinors), each call timed on the
    host around the synchronous library call (the new tensor's allocation included), against the
    reference's own functions on the host cores (one call each)."""
    import ctypes

    from rerdmft_b200 import _lib as L
    from rerdmft_b200 import synth

    lib = L.lib()
    out = {}
    inp = make_inputs()
    rng = np.random.default_rng(SEED + 5)
    C = np.ascontiguousarray(synth.random_orthogonal(N_AO, rng))
    dB = torch.from_numpy(inp["B"]).cuda()
    from rerdmft_b200.ri import RiStore

    st = RiStore(dB, nl=N_AO)
    dC = torch.from_numpy(C).cuda()
    o = L.opts(L.RR_MEM_DEVICE, sync=1)

    def build_nonrel():
        h = ctypes.c_void_p()
        L.check(lib.rr_mo_build_nonrel(st.handle, dC.data_ptr(), ctypes.byref(h), ctypes.byref(o)))
        return h

    h = build_nonrel()
    L.check(lib.rr_mo_destroy(h))
    times = []
    for _ in range(reps):
        t0 = time.perf_counter()
        h = build_nonrel()
        times.append(time.perf_counter() - t0)
        L.check(lib.rr_mo_destroy(h))
    best = min(times)
    flops = 4.0 * N_AUX * N_AO ** 3
    out["nonrel_spin"] = dict(workload=f"buildRiNonRelSpinMoEri n={N_AO} naux={N_AUX} (full C, FP64)",
                              seconds_per_build=best, algorithmic_gflop=flops / 1e9,
                              achieved_tflops=flops / best / 1e12,
                              frac_of_dgemm=(flops / best / 1e12 / fp64_peak) if fp64_peak else None,
                              note="host wall time of the synchronous call, the 2.05 GB output allocation included")

    # Device time of the same build into an existing tensor (rr_mo_build_nonrel_into: no allocation), CUDA
    # events on the call's stream; B (2.05 GB) and the output are far larger than L2, so no flush.
    stream = torch.cuda.current_stream()
    od = L.opts(L.RR_MEM_DEVICE, sync=0, stream=stream.cuda_stream)
    hm = build_nonrel()

    def device_seconds(prec, n_rep):
        od.precision = prec
        L.check(lib.rr_mo_build_nonrel_into(st.handle, dC.data_ptr(), hm, ctypes.byref(od)))
        torch.cuda.synchronize()
        ts = []
        for _ in range(n_rep):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            L.check(lib.rr_mo_build_nonrel_into(st.handle, dC.data_ptr(), hm, ctypes.byref(od)))
            e1.record(stream)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1) / 1e3)
        return float(np.median(ts))

    t64 = device_seconds(L.RR_PREC_FP64, reps)
    out["nonrel_spin"]["device_seconds_per_rebuild"] = t64
    out["nonrel_spin"]["device_frac_of_dgemm"] = (flops / t64 / 1e12 / fp64_peak) if fp64_peak else None
    b64 = np.empty((N_AUX, N_AO * N_AO))
    L.check(lib.rr_mo_copy_tensor(hm, b64.ctypes.data, ctypes.byref(L.opts())))
    tmx = device_seconds(L.RR_PREC_MIXED, 3 * reps)
    bmx = np.empty_like(b64)
    L.check(lib.rr_mo_copy_tensor(hm, bmx.ctypes.data, ctypes.byref(L.opts())))
    L.check(lib.rr_mo_destroy(hm))
    hbm, _ = measured_peaks()
    pk = ROOT / "MEASURED_PEAKS.json"
    bf16_peak = json.loads(pk.read_text()).get("bf16_tflops", 1590.0) if pk.exists() else 1590.0
    ldq = (N_AO + 7) // 8 * 8
    # bytes: the split copy of B read, the split intermediate written and read, the FP64 tensor written
    moved = N_AUX * N_AO * ldq * 2 * 2 * 3 + N_AUX * N_AO * N_AO * 8
    tc_flops = 3 * flops  # three BF16 products per FP64-equivalent product
    err = float(np.abs(bmx - b64).max())
    out["nonrel_spin_mixed"] = dict(
        workload=f"buildRiNonRelSpinMoEri n={N_AO} naux={N_AUX} (full C, split-BF16 tcgen05, RR_PREC_MIXED)",
        device_seconds_per_rebuild=tmx, speedup_over_fp64_device=t64 / tmx,
        tensor_tflops=tc_flops / tmx / 1e12,
        frac_of_bf16_peak=(tc_flops / tmx / 1e12 / bf16_peak) if bf16_peak else None,
        hbm_gbs=moved / tmx / 1e9, frac_of_hbm=(moved / tmx / 1e9 / hbm) if hbm else None,
        algorithmic_bytes=moved, bf16_mma_flops=tc_flops,
        max_abs_minus_fp64=err, rel_to_max=err / float(np.abs(b64).max()),
        kernel="umma_mo_kernel (two launches: B^P C split, then C^T (B^P C) in FP64)")
    del b64, bmx
    if want_cpu:
        from oracle import ref

        if ref.available():
            ref.set_threads(os.cpu_count() or 1)
            t0 = time.perf_counter()
            Bref = ref.nonrel_mo_build(inp["B"], C)
            dt = time.perf_counter() - t0
            h = build_nonrel()
            got = np.empty((N_AUX, N_AO * N_AO))
            L.check(lib.rr_mo_copy_tensor(h, got.ctypes.data, ctypes.byref(L.opts())))
            L.check(lib.rr_mo_destroy(h))
            out["nonrel_spin"]["reference_cpu"] = dict(seconds_per_build=dt, cores=os.cpu_count() or 1,
                                                       cpu_model=cpu_model(),
                                                       sample="one full-size call of the reference "
                                                              "buildRiNonRelSpinMoEri")
            out["nonrel_spin"]["parity"] = dict(max_abs_minus_reference=float(np.abs(got - Bref).max()),
                                                tolerance=1e-10)
            del Bref, got
    st.close()
    del dB, dC, inp
    torch.cuda.empty_cache()

    s = synth.rkb_system(NL4, NS4, NAUX4, 2 * (NOCC4 // 2), seed=SEED + 11, box=20.0)
    # the functional stage's MO space: the positive-energy half of the RKB basis (no-pair), 400 spinors
    nt = s["n_rkb"] // 2
    c_ukb = np.ascontiguousarray(s["v_total"] @ synth.random_unitary(s["n_rkb"], rng)[:, :nt])
    st4 = RiStore(torch.from_numpy(s["B_LL"]).cuda(), torch.from_numpy(s["B_SS"]).cuda(), nl=NL4, ns=NS4)
    dc = torch.from_numpy(c_ukb).cuda()

    def build_ukb():
        h = ctypes.c_void_p()
        L.check(lib.rr_mo_build_ukb(st4.handle, dc.data_ptr(), nt, ctypes.byref(h), ctypes.byref(o)))
        return h

    h = build_ukb()
    L.check(lib.rr_mo_destroy(h))
    times = []
    for _ in range(3):
        t0 = time.perf_counter()
        h = build_ukb()
        times.append(time.perf_counter() - t0)
        L.check(lib.rr_mo_destroy(h))
    best = min(times)
    # per flavour f: T = c_f^dagger B_f^P (2 real products, 2 nt fs^2 each) and T c_f (complex, 8 nt^2 fs)
    fl = [NL4, NL4, NS4, NS4]
    flops = NAUX4 * sum(4.0 * nt * f * f + 8.0 * nt * nt * f for f in fl)
    out["ukb_4c"] = dict(workload=f"buildRiMoEri nl={NL4} ns={NS4} naux={NAUX4} n_total={nt} (complex, FP64)",
                         seconds_per_build=best, algorithmic_gflop=flops / 1e9, achieved_tflops=flops / best / 1e12,
                         frac_of_dgemm=(flops / best / 1e12 / fp64_peak) if fp64_peak else None,
                         note="host wall time of the synchronous call, the 2.56 GB output allocation included")
    # split BF16 (RR_PREC_MIXED): same host-wall timing (new tensor each call), error against the FP64 build
    om = L.opts(L.RR_MEM_DEVICE, precision=L.RR_PREC_MIXED, sync=1)

    def build_ukb_mixed():
        hh = ctypes.c_void_p()
        L.check(lib.rr_mo_build_ukb(st4.handle, dc.data_ptr(), nt, ctypes.byref(hh), ctypes.byref(om)))
        return hh

    h = build_ukb()
    b64 = np.empty((NAUX4, 2 * nt * nt))
    L.check(lib.rr_mo_copy_tensor(h, b64.ctypes.data, ctypes.byref(L.opts())))
    L.check(lib.rr_mo_destroy(h))
    h = build_ukb_mixed()
    L.check(lib.rr_mo_destroy(h))
    times = []
    for _ in range(3):
        t0 = time.perf_counter()
        h = build_ukb_mixed()
        times.append(time.perf_counter() - t0)
        if len(times) < 3:
            L.check(lib.rr_mo_destroy(h))
    bmx = np.empty_like(b64)
    L.check(lib.rr_mo_copy_tensor(h, bmx.ctypes.data, ctypes.byref(L.opts())))
    L.check(lib.rr_mo_destroy(h))
    tm = min(times)
    nu4 = 2 * NL4 + 2 * NS4
    # BF16 MMA work: step 1 per flavour 2 fs^2 (2 nt) per aux index, step 2 2 nt (2 nt) (2 nu), 3 products each
    mma = 3.0 * NAUX4 * (sum(2.0 * f * f * 2 * nt for f in fl) + 2.0 * nt * 2 * nt * 2 * nu4)
    err = float(np.abs(bmx - b64).max())
    out["ukb_4c_mixed"] = dict(
        workload=f"buildRiMoEri nl={NL4} ns={NS4} naux={NAUX4} n_total={nt} (complex, split-BF16 tcgen05, "
                 "RR_PREC_MIXED)",
        seconds_per_build=tm, speedup_over_fp64=best / tm, bf16_mma_tflop=mma / 1e12,
        tensor_tflops=mma / tm / 1e12, max_abs_minus_fp64=err, rel_to_max=err / float(np.abs(b64).max()),
        note="host wall time of the synchronous call, the 2.56 GB output allocation included")
    del b64, bmx
    if want_cpu:
        from oracle import ref

        if ref.available():
            t0 = time.perf_counter()
            ref.ri_mo_build(NL4, NS4, s["B_LL"], s["B_SS"], c_ukb)
            out["ukb_4c"]["reference_cpu"] = dict(seconds_per_build=time.perf_counter() - t0,
                                                  cores=os.cpu_count() or 1, cpu_model=cpu_model(),
                                                  sample="one full-size call of the reference buildRiMoEri")
    st4.close()
    del dc
    torch.cuda.empty_cache()
    return out


def orbital_optimization_block():
    """Functional-stage orbital optimisation (ADAM macro loop at fixed occupations) with and without
    the shipped learned preconditioner: a LiH-sized system (11 spatial orbitals, naux 48; two seeds
    standing in for the 1.6 / 4.0 Angstrom geometries) and a synthetic one with 120 spatial orbitals
    (naux 480), iterations and wall time to |dE| < 1e-8 Ha between macro-iterations.  The learned
    runs finish with plain ADAM (polish), so both energies come from the plain method; their
    macro-iteration counts include the polishing runs.  Both methods are also run at uniformly larger
    base learning rates (2, 4, 8 x the reference's 0.01); for each the best rate whose run reaches the
    default plain run's energy to 1e-7 Ha is reported, so the learned scales are compared with the
    best uniform step as well as with the default."""
    from rerdmft_b200 import orbopt, synth

    net = orbopt.load_default_preconditioner()
    out = {}
    for name, ns, naux, seeds in (("lih_sized_n11", 11, 48, (16, 40)), ("synthetic_n120", 120, 480, (120,))):
        for seed in seeds:
            r = {}
            runs = {"plain": {}, "learned": {}}
            for mode in ("plain", "learned"):
                for factor in (1, 2, 4, 8):
                    opt = orbopt.adam_default_options()
                    opt.learning_rate = 0.01 * factor
                    prob, eri = orbopt.problem_from_system(synth.functional_system(ns, naux, seed, nocc=2), options=opt)
                    res = orbopt.run_full_optimization(prob, preconditioner=net if mode == "learned" else None,
                                                       max_macro=200)
                    prob.close()
                    eri.close()
                    runs[mode][factor] = dict(learning_rate=opt.learning_rate,
                                              **{k: res[k] for k in ("macro_iterations", "scaled_macro_iterations",
                                                                     "adam_steps", "seconds", "energy", "converged")})
                r[mode] = runs[mode][1]
            e_ref = r["plain"]["energy"]
            for mode in ("plain", "learned"):
                ok = [v for v in runs[mode].values() if v["converged"] and abs(v["energy"] - e_ref) <= 1e-7]
                r[mode + "_best_rate"] = min(ok, key=lambda v: v["macro_iterations"]) if ok else None
            r["macro_reduction"] = 1.0 - r["learned"]["macro_iterations"] / r["plain"]["macro_iterations"]
            if r["plain_best_rate"] and r["learned_best_rate"]:
                r["macro_reduction_best_rates"] = (1.0 - r["learned_best_rate"]["macro_iterations"] /
                                                   r["plain_best_rate"]["macro_iterations"])
            r["learned_minus_plain_energy"] = r["learned"]["energy"] - r["plain"]["energy"]
            out[f"{name}_seed{seed}"] = r
    net.close()
    return out


def gnof_optimization_block():
    """GNOF FULL_OPTIMIZATION (rerdmft_b200.pnof: device ADAM orbital runs, host occupation steps over
    the gamma angles from the device J/K) on LiH-sized systems (11 spatial orbitals, naux 48, two
    occupied pairs each coupled with three virtual pairs; two seeds): macro-iterations and wall time to
    |dE| < 1e-8 Ha with plain ADAM and with the learned preconditioner, each at the reference's base
    rate and at 2, 4, 8 x that rate (the best run that reaches the default plain energy to 1e-7 Ha is
    reported beside the default)."""
    from rerdmft_b200 import mo, orbopt, pnof, synth

    net = orbopt.load_default_preconditioner()
    out = {}
    n, nocc, coupling = 11, 2, 4
    for seed in (16, 40):
        f = synth.functional_system(n, 48, seed, nocc=nocc)
        gem = pnof.nonrel_geminals(n, nocc, coupling)
        occ0 = pnof.occupations_of(gem, coupling, np.full(nocc * (coupling - 1), np.pi / 4), 2 * n)
        two = pnof.full_two_rdm(pnof.FUNCTIONALS["GNOF"], gem, occ0, 2 * n)
        runs = {"plain": {}, "learned": {}}
        for mode in runs:
            for factor in (1, 2, 4, 8):
                opt = orbopt.adam_default_options()
                opt.learning_rate = 0.01 * factor
                eri = mo.RiNonRelSpinMoEri.from_tensor(f["Bmo"], n)
                prob = orbopt.RotationProblem(eri, f["h"], occ0, two["two_rdm_h"], two["two_rdm_x"], two["pair_of"],
                                              two["two_rdm_l1"], two["two_rdm_l2"], options=opt)
                res = pnof.run_pnof_optimization(prob, "GNOF", gem, coupling,
                                                 preconditioner=net if mode == "learned" else None)
                prob.close()
                eri.close()
                runs[mode][factor] = dict(learning_rate=opt.learning_rate,
                                          **{k: res[k] for k in ("macro_iterations", "scaled_macro_iterations",
                                                                 "adam_steps", "seconds", "energy", "converged")})
        r = {"plain": runs["plain"][1], "learned": runs["learned"][1]}
        e_ref = r["plain"]["energy"]
        for mode in runs:
            ok = [v for v in runs[mode].values() if v["converged"] and abs(v["energy"] - e_ref) <= 1e-7]
            r[mode + "_best_rate"] = min(ok, key=lambda v: v["macro_iterations"]) if ok else None
        r["macro_reduction"] = 1.0 - r["learned"]["macro_iterations"] / r["plain"]["macro_iterations"]
        if r["plain_best_rate"] and r["learned_best_rate"]:
            r["macro_reduction_best_rates"] = (1.0 - r["learned_best_rate"]["macro_iterations"] /
                                               r["plain_best_rate"]["macro_iterations"])
        out[f"lih_sized_n11_seed{seed}"] = r
    net.close()
    return out


def water_cluster(waters: int):
    """(H2O)_waters / cc-pVDZ (Cartesian) on a cubic grid 3 Angstrom apart, with its PAUTO aux basis: the
    orbital basis, the aux basis (both normalised as the reference normalises them) and the geometry.
    The basis data are the fixture tests/golden/water_ccpvdz.npz (the reference's example basis file)."""
    from rerdmft_b200 import basis as bs

    z = np.load(ROOT / "tests" / "golden" / "water_ccpvdz.npz")
    sets = bs.basis_set_from_arrays(z["shell_element"], z["shell_l"], z["shell_nprim"], z["exponents"],
                                    z["coefficients"])
    mol = [(str(s), *map(float, xyz)) for s, xyz in zip(z["atom_symbol"], z["atom_xyz"])]
    k = int(np.ceil(waters ** (1.0 / 3.0) - 1e-9))
    geo = []
    for i in range(waters):
        sh = np.array([i % k, (i // k) % k, i // (k * k)]) * 3.0 * bs.ANGSTROM_TO_BOHR
        geo += [bs.Atom(s, x + sh[0], y + sh[1], zz + sh[2]) for s, x, y, zz in mol]
    orb = bs.build_molecular_basis(geo, sets)
    bs.normalize_cartesian_basis(orb)
    aux = bs.build_auto_auxiliary_basis(orb, "PAUTO")
    bs.normalize_cartesian_basis(aux)
    return orb, aux, geo


def lih_631g():
    """LiH / 6-31G at 1.5949 Angstrom with its PAUTO aux basis, and the RI Hartree-Fock energy the reference
    printed for it (fixture tests/golden/lih_631g.npz)."""
    from rerdmft_b200 import basis as bs

    z = np.load(ROOT / "tests" / "golden" / "lih_631g.npz")
    sets = bs.basis_set_from_arrays(z["shell_element"], z["shell_l"], z["shell_nprim"], z["exponents"],
                                    z["coefficients"])
    geo = [bs.Atom(str(s), *map(float, xyz)) for s, xyz in zip(z["atom_symbol"], z["atom_xyz"])]
    orb = bs.build_molecular_basis(geo, sets)
    bs.normalize_cartesian_basis(orb)
    aux = bs.build_auto_auxiliary_basis(orb, "PAUTO")
    bs.normalize_cartesian_basis(aux)
    return orb, aux, geo, int(z["nelec"]), float(z["e_hf_ri"])


def integrals_block(torch, hbm_peak, want_cpu: bool, waters: int = 8, reps: int = 3):
    """The device integral engine: the raw 3-centre integrals and the aux metric of (H2O)_waters / cc-pVDZ
    (PAUTO aux basis), device outputs, CUDA events; and, in the CPU leg, LiH / 6-31G against the numpy
    restatement (time and max relative difference) and its RI Hartree-Fock energy from device integrals and
    the device SCF loop against the reference's printed value."""
    import ctypes

    from rerdmft_b200 import _lib as L
    from rerdmft_b200 import basis as bs
    from rerdmft_b200 import integrals as gi

    lib = L.lib()
    orb, aux, _ = water_cluster(waters)
    n, na = len(orb), len(aux)
    co, ca = gi._CBasis(orb), gi._CBasis(aux)
    raw = torch.empty((na, n * n), dtype=torch.float64, device="cuda")
    M = torch.empty((na, na), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    o = L.opts(L.RR_MEM_DEVICE, stream=stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    ms_raw = timed(lambda: L.check(lib.rr_int_three_center_raw(ctypes.byref(co.c), ctypes.byref(ca.c), raw.data_ptr(),
                                                               ctypes.byref(o))))
    ms_m = timed(lambda: L.check(lib.rr_int_aux_metric(ctypes.byref(ca.c), M.data_ptr(), ctypes.byref(o))))
    shells_o = [(orb[f].l, len(orb[f].exponents)) for f, _ in bs.group_into_shells(orb)]
    shells_a = [(aux[f].l, len(aux[f].exponents)) for f, _ in bs.group_into_shells(aux)]
    prim_a = sum(p for _, p in shells_a)
    triples = sum(shells_o[i][1] * shells_o[j][1] for i in range(len(shells_o)) for j in range(i, len(shells_o))) * prim_a
    raw_bytes = 8.0 * na * n * n
    out = dict(workload=f"(H2O)_{waters} / cc-pVDZ (Cartesian), PAUTO aux basis: raw (pq|P) and (P|Q), FP64",
               n=n, naux=na, raw_gb=raw_bytes / 1e9, ms_raw=ms_raw, ms_metric=ms_m,
               primitive_triples=triples, primitive_triples_per_s=triples / (ms_raw / 1e3),
               raw_write_gbs=raw_bytes / (ms_raw / 1e3) / 1e9,
               write_floor_ms=(raw_bytes / (hbm_peak * 1e9) * 1e3) if hbm_peak else None,
               note="compute-bound (FP64 Hermite recurrences); the write floor is the raw tensor at measured HBM")
    del raw, M
    torch.cuda.empty_cache()
    if want_cpu:
        sys.path.insert(0, str(ROOT))
        from oracle import integrals_oracle as io
        from oracle import ri_oracle as ro
        from rerdmft_b200 import ri, scf

        lorb, laux, geo, nelec, e_ref = lih_631g()
        t0 = time.perf_counter()
        raw_ref = io.three_center_raw(lorb, laux)
        cpu_s = time.perf_counter() - t0
        t0 = time.perf_counter()
        raw_dev = gi.threeCenterIntegralsRaw(lorb, laux)
        dev_s = time.perf_counter() - t0
        S = io.overlap_matrix(lorb)
        ch = [(bs.atomic_number(a.symbol), (a.x, a.y, a.z)) for a in geo]
        h = io.kinetic_matrix(lorb) + io.nuclear_attraction_matrix(lorb, ch)
        X = ro.canonical_orthogonalize(S, 1e-6)
        store, rep = gi.store_from_basis(lorb, laux, 1e-10)
        src = ri.RiNonRelEriSource(len(lorb), None, X, S, store=store)
        w, u = np.linalg.eigh(X.T @ h @ X)
        c = X @ u[:, :nelec // 2]
        r = scf.runNonRelativisticHartreeFock(src, h, X, 2.0 * c @ c.T, nelec)
        e = r["energy"] + bs.nuclear_repulsion(geo)
        store.close()
        out["parity"] = dict(
            workload="LiH / 6-31G (n = 11) with its PAUTO aux basis (naux = 106)",
            raw_max_rel_vs_restatement=float(np.abs(raw_dev - raw_ref).max() / np.abs(raw_ref).max()),
            ri_hf_energy=e, reference_energy=e_ref, energy_minus_reference=e - e_ref,
            reference="the reference's printed RI-HF energy (libcint integrals), examples/reference.yaml",
            metric_kept=rep["n_kept"], metric_dropped=rep["n_dropped"])
        out["cpu_baseline"] = dict(kind="port", cores=1, seconds=cpu_s, device_call_seconds=dev_s,
                                   sample="LiH / 6-31G raw tensor by the numpy McMurchie-Davidson restatement (the "
                                          "reference's libcint is not available here)")
    return out


def x2c_batch_problems(count: int = 64):
    """The batched X2C-HF geometry scan: `count` instances with uneven nl in [20, 120] (seeded), naux = 4 nl,
    4 or 14 electrons (LiH- / CO-like) alternating, one handle each (uploaded here)."""
    from rerdmft_b200 import ri, synth

    rng = np.random.default_rng(SEED + 44)
    sizes = rng.integers(20, 121, size=count)
    probs, systems = [], []
    for k, nl in enumerate(sizes):
        sysd = synth.x2c_system(int(nl), 4 * int(nl), 4 if k % 2 == 0 else 14, seed=SEED + 100 + k)
        src = ri.RiX2cEriSource(int(nl), sysd["B"], sysd["X"], sysd["S"])
        src.store  # upload outside the timed region
        systems.append(sysd)
        probs.append(dict(eri=src, h_x2c=sysd["h"], x_large=sysd["X"], initial_density=sysd["P0"],
                          n_electrons=sysd["n_electrons"]))
    return sizes, probs, systems


def x2c_batch_block(want_cpu: bool, count: int = 64, workers: int = 16):
    """Batched X2C-HF geometry scan (x2c_batch_problems), each instance converged to 1e-8 Ha: one after
    another (workers = 1), concurrently on host threads (rr_scf_run_x2c_batch), and in lockstep as one
    grouped program (rr_scf_run_x2c_grouped: one grouped launch per phase per iteration for all instances,
    autotuned tiles; the first run tunes the shapes, the timed run uses the cache)."""
    from rerdmft_b200 import scf

    sizes, probs, systems = x2c_batch_problems(count)
    scf.runX2CHartreeFockScfBatch(probs, workers=workers)  # warm-up: every handle's first-call allocations
    t0 = time.perf_counter()
    seq = scf.runX2CHartreeFockScfBatch(probs, workers=1)
    t_seq = time.perf_counter() - t0
    t0 = time.perf_counter()
    par = scf.runX2CHartreeFockScfBatch(probs, workers=workers)
    t_par = time.perf_counter() - t0
    tune = {}
    scf.runX2CHartreeFockScfBatch(probs, mode="grouped", stats=tune)  # tunes every new shape
    st = {}
    t0 = time.perf_counter()
    grp = scf.runX2CHartreeFockScfBatch(probs, mode="grouped", stats=st)
    t_grp = time.perf_counter() - t0
    out = dict(workload=f"{count} X2C-HF instances, nl in [20, 120] (uneven), naux = 4 nl, 4 / 14 electrons, FP64",
               seconds_one_after_another=t_seq, seconds_concurrent=t_par, workers=workers,
               instances_per_s=count / t_par, converged=int(sum(r["converged"] for r in par)),
               iterations_total=int(sum(r["iterations"] for r in par)),
               max_energy_difference_sequential_vs_concurrent=float(max(abs(a["energy"] - b["energy"])
                                                                      for a, b in zip(seq, par))),
               grouped=dict(seconds=t_grp, instances_per_s=count / t_grp,
                            converged=int(sum(r["converged"] for r in grp)),
                            lockstep_iterations=st["iterations"], launches_total=st["launches_total"],
                            launches_setup=st["launches_setup"],
                            launches_max_iteration=st["launches_max_iteration"],
                            instances_first_iteration_grouped=st["grouped_instances_first"],
                            max_energy_difference_vs_concurrent=float(max(abs(a["energy"] - b["energy"])
                                                                          for a, b in zip(grp, par))),
                            autotune=dict(seconds_first_run=tune["autotune_seconds"],
                                          shapes_cached=st["autotune_entries"],
                                          seconds_timed_run=st["autotune_seconds"])))
    if want_cpu:
        from oracle import ref

        if ref.available():
            ref.set_threads(os.cpu_count() or 1)
            sample = list(range(0, count, 8))
            t0 = time.perf_counter()
            for k in sample:
                ref.x2c_scf(systems[k])
            dt = time.perf_counter() - t0
            share = sum(int(sizes[k]) ** 3 for k in sample) / sum(int(x) ** 3 for x in sizes)
            out["reference_cpu"] = dict(seconds_sample=dt, sample=f"instances {sample} (every 8th)",
                                        cores=os.cpu_count() or 1,
                                        seconds_all_estimated_by_nl3=dt / share)
    for p in probs:
        p["eri"].store.close()
    return out


def scf_times(torch, want_cpu: bool):
    """Time to an energy change below 1e-8 Ha on one GPU: FP64 loop vs mixed loop (incremental
    split-BF16 exchange, one FP64 build of the final density), plus the reference's own SCF loop on the
    host cores."""
    from rerdmft_b200 import ri, scf

    s = make_scf_system()
    src = ri.RiNonRelEriSource(N_AO, s["B"], s["X"], s["S"])
    kw = dict(energy_tolerance=1e-8, density_tolerance=1e-6)
    out = {}
    for prec in ("fp64", "mixed"):
        scf.runNonRelativisticHartreeFock(src, s["h"], s["X"], s["D0"], s["n_electrons"], precision=prec, **kw)  # warm
        best = None
        for _ in range(3):
            r = scf.runNonRelativisticHartreeFock(src, s["h"], s["X"], s["D0"], s["n_electrons"], precision=prec, **kw)
            if best is None or r["seconds"] < best["seconds"]:
                best = r
        out[prec] = dict(seconds=best["seconds"], energy=best["energy"], iterations=best["iterations"],
                         converged=best["converged"], mixed_iterations=best["mixed_iterations"],
                         fp64_iterations=best["fp64_iterations"])
    out["mixed_over_fp64_time"] = out["mixed"]["seconds"] / out["fp64"]["seconds"]
    out["mixed_minus_fp64_energy"] = out["mixed"]["energy"] - out["fp64"]["energy"]
    if want_cpu:
        from oracle import ref

        if ref.available():
            ref.set_threads(os.cpu_count() or 1)
            t0 = time.perf_counter()
            rr = ref.nonrel_scf(s, e_tol=1e-8, d_tol=1e-6)
            out["reference_cpu"] = dict(seconds=time.perf_counter() - t0, energy=rr["energy"],
                                        iterations=rr["iterations"], cores=os.cpu_count() or 1)
            out["gpu_fp64_minus_reference_energy"] = out["fp64"]["energy"] - rr["energy"]
    src.store.close()
    return out


# Relativistic time-to-convergence systems (the 4-component shapes of the Kramers-restricted DHF
# configuration, and an X2C-HF system of 400 spinors): the synthetic generator's two-electron part
# is scaled (B by the factor, so J and K by its square) so that the FP64 loops need several
# iterations, as molecular SCFs do.
X2C_NL, X2C_NAUX, X2C_NE, X2C_GAP, X2C_B = 200, 1000, 80, 1.5, 6.0
DHF_GAP, DHF_B = 0.4, 3.0


def rel_scf_times(want_cpu: bool, rkb_ref_build_s=None):
    """Time to an energy change below 1e-8 Ha on one GPU for X2C-HF and 4c-DHF: the FP64 loop against
    the mixed loop (incremental split-BF16 exchange, one FP64 build of the final density), best of three
    runs each, with per-phase device times; the reference's CPU time is one of its own Fock builds of the
    same system times the FP64 iteration count (its loop spends nearly all its time in those builds)."""
    from rerdmft_b200 import _lib as L
    from rerdmft_b200 import ri, scf, synth

    def compare(run, src):
        L.check(L.lib().rr_ri_set_profiling(src.store.handle, 1))
        out = {}
        for prec in ("fp64", "mixed"):
            run(prec)  # warm-up (builds the split-BF16 operands once)
            best = None
            for _ in range(3):
                r = run(prec)
                if best is None or r["seconds"] < best["seconds"]:
                    best = r
            out[prec] = dict(seconds=best["seconds"], energy=best["energy"], iterations=best["iterations"],
                             converged=best["converged"], mixed_iterations=best["mixed_iterations"],
                             fp64_iterations=best["fp64_iterations"],
                             phase_ms={k: round(v, 3) for k, v in best["phase_ms"].items()})
        out["mixed_over_fp64_time"] = out["mixed"]["seconds"] / out["fp64"]["seconds"]
        out["mixed_minus_fp64_energy"] = out["mixed"]["energy"] - out["fp64"]["energy"]
        return out

    res = {}
    s = synth.x2c_system(X2C_NL, X2C_NAUX, X2C_NE, seed=SEED + 21, box=20.0, gap=X2C_GAP)
    B = s["B"] * X2C_B
    src = ri.RiX2cEriSource(X2C_NL, B, s["X"], s["S"])
    res["x2c_hf"] = compare(lambda prec: scf.runX2CHartreeFockScf(s["h"], src, s["X"], s["P0"], X2C_NE, precision=prec),
                            src)
    res["x2c_hf"]["workload"] = (f"X2C-HF nl={X2C_NL} ({2 * X2C_NL} spinors) naux={X2C_NAUX} {X2C_NE} electrons, "
                                 f"core gap {X2C_GAP} Ha, B x {X2C_B}")
    if want_cpu:
        from oracle import ref

        if ref.available():
            ref.set_threads(os.cpu_count() or 1)
            t0 = time.perf_counter()
            ref.x2c_fock(s["h"], B, s["P0"], s["S"], s["X"])
            dt = time.perf_counter() - t0
            res["x2c_hf"]["reference_cpu"] = dict(
                seconds_estimate=dt * res["x2c_hf"]["fp64"]["iterations"], seconds_per_build=dt,
                cores=os.cpu_count() or 1, sample="one reference x2cFockMatrix of this system x the FP64 iteration count")
    src.store.close()
    del B, s
    s = synth.rkb_system(NL4, NS4, NAUX4, 2 * (NOCC4 // 2), seed=SEED + 11, box=20.0, gap=DHF_GAP)
    src = ri.RiDirectEriSource(NL4, NS4, s["B_LL"] * DHF_B, s["B_SS"] * DHF_B, s["v_total"], s["s_full"], s["x_full"])
    ne = 2 * (NOCC4 // 2)
    res["dhf_4c"] = compare(lambda prec: scf.runDiracHartreeFockScf(s["h"], src, s["x_full"], s["P0"], ne,
                                                                      precision=prec), src)
    res["dhf_4c"]["workload"] = (f"4c-DHF nl={NL4} ns={NS4} naux={NAUX4} {ne} electrons (RKB basis {4 * NL4}), "
                                 f"core gap {DHF_GAP} Ha, B x {DHF_B}")
    if want_cpu and rkb_ref_build_s:
        res["dhf_4c"]["reference_cpu"] = dict(
            seconds_estimate=rkb_ref_build_s * res["dhf_4c"]["fp64"]["iterations"], seconds_per_build=rkb_ref_build_s,
            cores=os.cpu_count() or 1,
            sample="the reference rkbFockMatrix time of the 4c Fock-build block (same shapes) x the FP64 iteration count")
    src.store.close()
    return res


def max_over_ranks(pg, seconds: float, device: str) -> float:
    """The job's time: the slowest rank's (all-reduce MAX of one float; unchanged with one rank)."""
    if pg is None:
        return seconds
    import torch

    tt = torch.tensor([seconds], dtype=torch.float64, device=device)
    pg.all_reduce(tt, op=pg.ReduceOp.MAX)
    return float(tt.item())


def replica_throughput(world_size: int, steps: int, seconds: float) -> float:
    """Whole-job builds/s: every replica runs `steps` builds within the slowest rank's time."""
    return world_size * steps / seconds


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def fp64_gemm_peak(torch) -> float:
    """Measured FP64 tensor-core peak on this GPU: cuBLAS DGEMM 8192^3 (TFLOP/s, best of 5)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    del a, b
    return 2.0 * n ** 3 / best / 1e12


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d.get("hbm_gbs", 6650.0), "MEASURED_PEAKS.json"
    return 6650.0, "fallback"


def cpu_reference_rate(inp, seconds: float = 15.0):
    """The reference's own nonRelFockMatrix (oracle/_ref, compiled from its sources) on the same
    inputs, all host cores (OMP threads, serial BLAS inside, as the reference expects)."""
    from oracle import ref

    if not ref.available():
        return None, None
    cores = os.cpu_count() or 1
    ref.set_threads(cores)
    t0 = time.perf_counter()
    F_ref = ref.nonrel_fock(inp["h"], inp["B"], inp["D"], inp["S"], inp["X"])
    first = time.perf_counter() - t0
    reps = max(1, min(20, int(seconds / max(first, 1e-3))))
    best = first
    for _ in range(reps):
        t0 = time.perf_counter()
        ref.nonrel_fock(inp["h"], inp["B"], inp["D"], inp["S"], inp["X"])
        best = min(best, time.perf_counter() - t0)
    return dict(value=1.0 / best, unit=UNIT, cores=cores, cpu_model=cpu_model(), kind="reference",
                sample=f"full workload (n={N_AO}, naux={N_AUX}, nocc={N_OCC}), best of {reps + 1} calls of the "
                       f"reference nonRelFockMatrix compiled from its sources, OMP_NUM_THREADS={cores}"), F_ref


def run_reference(args):
    ws, rank, _ = dist_env()
    base = dict(metric=METRIC, unit=UNIT, n_gpus=args.gpus, steps=args.steps, warmup=args.warmup,
                higher_is_better=True, scaling="weak", vs_baseline=None, dtype="f64", data="synthetic",
                impl="reference", config=bench_config(args.gpus))
    if rank != 0:
        return
    from oracle import ref

    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/librrref.so not built"}))
        return
    inp = make_inputs()
    cores = os.cpu_count() or 1
    ref.set_threads(cores)
    # Every warm-up and timed step is one full-size call; if one call is so slow that the run would
    # exceed about four minutes, fewer steps run and the line says how many.
    t0 = time.perf_counter()
    ref.nonrel_fock(inp["h"], inp["B"], inp["D"], inp["S"], inp["X"])
    first = time.perf_counter() - t0
    budget = max(1, int(240.0 / max(first, 1e-3)))
    warmup = max(0, min(args.warmup - 1, budget // 4))
    steps = max(1, min(args.steps, budget - warmup - 1))
    for _ in range(warmup):
        ref.nonrel_fock(inp["h"], inp["B"], inp["D"], inp["S"], inp["X"])
    t0 = time.perf_counter()
    for _ in range(steps):
        ref.nonrel_fock(inp["h"], inp["B"], inp["D"], inp["S"], inp["X"])
    dt = time.perf_counter() - t0
    v = steps / dt
    base.update(steps=steps, warmup=warmup + 1, value=v, ms_per_step=1e3 * dt / steps,
                cpu_baseline=dict(value=v, unit=UNIT, cores=cores, cpu_model=cpu_model(), kind="reference",
                                  sample=f"{steps} timed full-size calls after {warmup + 1} warm-up calls of the "
                                         f"reference nonRelFockMatrix compiled from its sources, "
                                         f"OMP_NUM_THREADS={cores}"),
                e2e=dict(value=v, unit=UNIT, h2d_bytes_per_step=0, d2h_bytes_per_step=0))
    print(json.dumps(base))


def run_case(args):
    """Single workloads for profiling and kernel timing (one GPU, device-resident inputs, CUDA events):
    headline      the FP64 nonrel Fock build of the headline workload only (no extra blocks);
    mixed_exchange  the split-BF16 tcgen05 exchange K = sum_P (Ct B^P)^T (Ct B^P) at n=400, naux=1600,
                  nocc=40 (rr_ri_jk_occupied, RR_PREC_MIXED; J stays FP64);
    rkb_mixed     the 4c RKB Fock build of the Kramers-restricted DHF shapes with the split-BF16 exchange,
                  full then incremental (nl=200, ns=600, naux=1000, 40 spinors);
    rkb_fp64      the same 4c RKB Fock build in FP64 (the 4c Fock-build workload of the bench line);
    x2c_mixed     the X2C Fock build with the split-BF16 exchange, full then incremental (nl=200,
                  naux=1000, 80 electrons);
    x2c_batch     the lockstep grouped X2C-HF scan (64 uneven instances), tuned then timed once;
    integrals     the raw 3-centre integrals and the aux metric of (H2O)_8 / cc-pVDZ with its PAUTO aux basis
                  (n = 200, naux = 2856; RR_WATERS=<k> for another cluster), device outputs;
    mo_mixed      the split-BF16 MO transform B_mo^P = C^T B^P C rebuilt into one tensor (n = 400, naux = 1600;
                  RR_MO_NAUX=<k> for fewer aux rows), and the FP64 build of the same tensor (mo_fp64)."""
    import ctypes

    import torch

    from rerdmft_b200 import _lib as L
    from rerdmft_b200 import ri, synth

    torch.cuda.set_stream(torch.cuda.Stream())  # events and library calls on one real stream
    lib = L.lib()
    stream = torch.cuda.current_stream().cuda_stream
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(step, steps, warmup):
        for _ in range(warmup):
            step()
        torch.cuda.synchronize()
        e0.record()
        for _ in range(steps):
            step()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    out = dict(case=args.case, steps=args.steps, warmup=args.warmup)
    if args.case == "integrals":
        from rerdmft_b200 import integrals as gi

        waters = int(os.environ.get("RR_WATERS", "8"))
        orb, aux, _ = water_cluster(waters)
        n, na = len(orb), len(aux)
        co, ca = gi._CBasis(orb), gi._CBasis(aux)
        raw = torch.empty((na, n * n), dtype=torch.float64, device="cuda")
        M = torch.empty((na, na), dtype=torch.float64, device="cuda")
        o = L.opts(L.RR_MEM_DEVICE, stream=stream)
        ms_raw = timed(lambda: L.check(lib.rr_int_three_center_raw(ctypes.byref(co.c), ctypes.byref(ca.c),
                                                                   raw.data_ptr(), ctypes.byref(o))),
                       args.steps, args.warmup)
        ms_m = timed(lambda: L.check(lib.rr_int_aux_metric(ctypes.byref(ca.c), M.data_ptr(), ctypes.byref(o))),
                     args.steps, args.warmup)
        out.update(workload=f"(H2O)_{waters} cc-pVDZ raw 3-centre integrals n={n} naux={na}", ms_raw=ms_raw,
                   ms_metric=ms_m, raw_gb=na * n * n * 8 / 1e9)
        print(json.dumps(out))
        return
    if args.case in ("mo_mixed", "mo_fp64"):
        na = int(os.environ.get("RR_MO_NAUX", str(N_AUX)))
        B = synth.ri_tensor(N_AO, na, SEED, box=20.0)
        C = synth.random_orthogonal(N_AO, np.random.default_rng(SEED + 5))
        st = ri.RiStore(torch.from_numpy(B).cuda(), nl=N_AO)
        dC = torch.from_numpy(C).cuda()
        prec = L.RR_PREC_MIXED if args.case == "mo_mixed" else L.RR_PREC_FP64
        h = ctypes.c_void_p()
        L.check(lib.rr_mo_build_nonrel(st.handle, dC.data_ptr(), ctypes.byref(h),
                                       ctypes.byref(L.opts(L.RR_MEM_DEVICE, precision=prec))))
        o = L.opts(L.RR_MEM_DEVICE, precision=prec, stream=stream, sync=0)
        ms = timed(lambda: L.check(lib.rr_mo_build_nonrel_into(st.handle, dC.data_ptr(), h, ctypes.byref(o))),
                   args.steps, args.warmup)
        L.check(lib.rr_mo_destroy(h))
        st.close()
        out.update(workload=f"buildRiNonRelSpinMoEri n={N_AO} naux={na} ({args.case})", ms_per_build=ms,
                   gflop_fp64_equivalent=4.0 * na * N_AO ** 3 / 1e9)
        print(json.dumps(out))
        return
    if args.case == "x2c_batch":
        from rerdmft_b200 import scf

        _, probs, _ = x2c_batch_problems()
        tune, st = {}, {}
        scf.runX2CHartreeFockScfBatch(probs, mode="grouped", stats=tune)
        t0 = time.perf_counter()
        res = scf.runX2CHartreeFockScfBatch(probs, mode="grouped", stats=st)
        out.update(workload="64 X2C-HF instances, grouped lockstep", seconds=time.perf_counter() - t0,
                   converged=int(sum(r["converged"] for r in res)), stats=st, tuning_run=tune)
        for p in probs:
            p["eri"].store.close()
        print(json.dumps(out))
        return
    if args.case in ("headline", "mixed_exchange"):
        inp = make_inputs()
        dev = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in inp.items()}
        store = ri.RiNonRelEriSource(N_AO, dev["B"], dev["X"], dev["S"]).store
        if args.case == "headline":
            F = torch.empty((N_AO, N_AO), dtype=torch.float64, device="cuda")
            o = L.opts(L.RR_MEM_DEVICE, stream=stream, sync=0)
            ms = timed(lambda: L.check(lib.rr_ri_fock_nonrel(store.handle, dev["h"].data_ptr(), dev["D"].data_ptr(),
                                                             dev["S"].data_ptr(), dev["X"].data_ptr(), N_AO,
                                                             F.data_ptr(), ctypes.byref(o))), args.steps, args.warmup)
            out.update(workload=f"FP64 nonrel Fock build n={N_AO} naux={N_AUX} nocc={N_OCC}", ms_per_build=ms)
        else:
            J = torch.empty((N_AO, N_AO), dtype=torch.float64, device="cuda")
            K = torch.empty_like(J)
            C = dev["C"].contiguous()
            o = L.opts(L.RR_MEM_DEVICE, precision=L.RR_PREC_MIXED, stream=stream, sync=0)
            ms = timed(lambda: L.check(lib.rr_ri_jk_occupied(store.handle, C.data_ptr(), N_OCC, J.data_ptr(),
                                                             K.data_ptr(), ctypes.byref(o))), args.steps, args.warmup)
            out.update(workload=f"split-BF16 J/K n={N_AO} naux={N_AUX} nocc={N_OCC}", ms_per_call=ms)
        store.sync()
    elif args.case in ("rkb_mixed", "rkb_fp64"):
        s = synth.rkb_system(NL4, NS4, NAUX4, 2 * (NOCC4 // 2), seed=SEED + 11, box=20.0)
        dev = {k: torch.from_numpy(np.ascontiguousarray(s[k])).cuda()
               for k in ("B_LL", "B_SS", "v_total", "s_full", "x_full", "h", "P0")}
        store = ri.RiDirectEriSource(NL4, NS4, dev["B_LL"], dev["B_SS"], dev["v_total"], dev["s_full"],
                                     dev["x_full"]).store
        n_rkb = s["n_rkb"]
        F = torch.empty((n_rkb, n_rkb), dtype=torch.complex128, device="cuda")
        x = dev["x_full"]

        def step(incremental):
            o = L.opts(L.RR_MEM_DEVICE, precision=L.RR_PREC_MIXED, stream=stream, sync=0, incremental=incremental)
            L.check(lib.rr_ri_fock_rkb(store.handle, dev["h"].data_ptr(), dev["v_total"].data_ptr(), n_rkb,
                                       dev["s_full"].data_ptr(), x.data_ptr(), x.shape[1], dev["P0"].data_ptr(),
                                       F.data_ptr(), ctypes.byref(o)))

        if args.case == "rkb_fp64":
            o64 = L.opts(L.RR_MEM_DEVICE, stream=stream, sync=0)
            ms = timed(lambda: L.check(lib.rr_ri_fock_rkb(store.handle, dev["h"].data_ptr(), dev["v_total"].data_ptr(),
                                                          n_rkb, dev["s_full"].data_ptr(), x.data_ptr(), x.shape[1],
                                                          dev["P0"].data_ptr(), F.data_ptr(), ctypes.byref(o64))),
                       args.steps, args.warmup)
            out.update(workload=f"FP64 rkbFockMatrix nl={NL4} ns={NS4} naux={NAUX4} nocc={NOCC4}", ms_per_build=ms)
        else:
            full = timed(lambda: step(0), args.steps, args.warmup)
            incr = timed(lambda: step(1), args.steps, args.warmup)
            out.update(workload=f"mixed rkbFockMatrix nl={NL4} ns={NS4} naux={NAUX4} nocc={NOCC4}", ms_full=full,
                       ms_incremental=incr)
        store.sync()
    elif args.case == "x2c_mixed":
        s = synth.x2c_system(X2C_NL, X2C_NAUX, X2C_NE, seed=SEED + 21, box=20.0, gap=X2C_GAP)
        dev = {k: torch.from_numpy(np.ascontiguousarray(s[k])).cuda() for k in ("B", "h", "S", "X", "P0")}
        store = ri.RiX2cEriSource(X2C_NL, dev["B"], dev["X"], dev["S"]).store
        n = 2 * X2C_NL
        F = torch.empty((n, n), dtype=torch.complex128, device="cuda")
        X = dev["X"]

        def step(incremental):
            o = L.opts(L.RR_MEM_DEVICE, precision=L.RR_PREC_MIXED, stream=stream, sync=0, incremental=incremental)
            L.check(lib.rr_ri_fock_x2c(store.handle, dev["h"].data_ptr(), dev["P0"].data_ptr(), dev["S"].data_ptr(),
                                       X.data_ptr(), X.shape[1], F.data_ptr(), ctypes.byref(o)))

        full = timed(lambda: step(0), args.steps, args.warmup)
        incr = timed(lambda: step(1), args.steps, args.warmup)
        out.update(workload=f"mixed x2cFockMatrix nl={X2C_NL} naux={X2C_NAUX} {X2C_NE} electrons", ms_full=full,
                   ms_incremental=incr)
        store.sync()
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--case", default=None, choices=["headline", "mixed_exchange", "rkb_mixed", "rkb_fp64", "x2c_mixed",
                                                    "x2c_batch", "integrals", "mo_mixed", "mo_fp64"],
                    help="run one workload for profiling instead of the bench line")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if args.impl == "reference":
        return run_reference(args)
    if args.case:
        return run_case(args)

    import torch

    from rerdmft_b200 import _lib as L
    from rerdmft_b200 import ri

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    # A real stream: the library runs on the stream it is given, and the CUDA events below are recorded
    # on the same one (torch's legacy default stream has handle 0, which the library reads as "its own").
    torch.cuda.set_stream(torch.cuda.Stream())
    pg = None
    if ws > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    inp = make_inputs()
    dev = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in inp.items() if k != "C"}
    src = ri.RiNonRelEriSource(N_AO, dev["B"], dev["X"], dev["S"])
    store = src.store
    lib = L.lib()
    F = torch.empty((N_AO, N_AO), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    o = L.opts(L.RR_MEM_DEVICE, stream=stream, sync=0)
    import ctypes

    def step():
        L.check(lib.rr_ri_fock_nonrel(store.handle, dev["h"].data_ptr(), dev["D"].data_ptr(), dev["S"].data_ptr(),
                                      dev["X"].data_ptr(), N_AO, F.data_ptr(), ctypes.byref(o)))

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    l0 = lib.rr_kernel_launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    launches = lib.rr_kernel_launches() - l0
    t = e0.elapsed_time(e1) / 1e3
    t = max_over_ranks(pg, t, "cuda")
    clk = clocks.stop()
    store.sync()
    value = replica_throughput(ws, args.steps, t)

    # Phase times from profiled calls (events inside the library, same stream).
    L.check(lib.rr_ri_set_profiling(store.handle, 1))
    acc = {}
    nprof = 5
    for _ in range(nprof):
        step()
        tm = L.Timings()
        L.check(lib.rr_ri_get_timings(store.handle, ctypes.byref(tm)))
        for k, v in tm.as_dict().items():
            acc[k] = acc.get(k, 0.0) + v / nprof
    L.check(lib.rr_ri_set_profiling(store.handle, 0))

    # End to end through the public API with host buffers (pinned): h, D, S, X in, F out.
    hp = {k: torch.from_numpy(np.ascontiguousarray(inp[k])).pin_memory() for k in ("h", "D", "S", "X")}
    Fh = torch.empty((N_AO, N_AO), dtype=torch.float64).pin_memory()
    oh = L.opts(L.RR_MEM_HOST, stream=stream, sync=1)

    def step_host():
        L.check(lib.rr_ri_fock_nonrel(store.handle, hp["h"].data_ptr(), hp["D"].data_ptr(), hp["S"].data_ptr(),
                                      hp["X"].data_ptr(), N_AO, Fh.data_ptr(), ctypes.byref(oh)))

    for _ in range(3):
        step_host()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    e0.record()
    for _ in range(args.steps):
        step_host()
    e1.record()
    torch.cuda.synchronize()
    te = e0.elapsed_time(e1) / 1e3
    te = max_over_ranks(pg, te, "cuda")
    e2e = dict(value=replica_throughput(ws, args.steps, te), unit=UNIT, h2d_bytes_per_step=4 * N_AO * N_AO * 8,
               d2h_bytes_per_step=N_AO * N_AO * 8)

    # Roofline of the dominant kernel group.
    hbm_peak, hbm_src = measured_peaks()
    fp64_peak = fp64_gemm_peak(torch) if rank == 0 else None
    ht_flops = 2.0 * N_AUX * N_OCC * N_AO * N_AO
    # The exchange SYRK computes only the upper 80 x 80 output tiles of the symmetric K (15 of 25 at
    # n = 400) and mirrors the rest: executed flops, not the full 2*naux*nocc*n^2 count.
    syrk_tile = 80
    syrk_nt = -(-N_AO // syrk_tile)
    syrk_flops = 2.0 * N_AUX * N_OCC * (syrk_nt * (syrk_nt + 1) // 2) * syrk_tile * syrk_tile
    j_bytes = 2.0 * N_AUX * N_AO * N_AO * 8  # algorithmic: two passes over B
    # both passes stream the packed upper triangles of B (from the top of the build, beside the recovery)
    j_bytes_streamed = 2.0 * N_AUX * (-(-(N_AO * (N_AO + 1) // 2) // 32) * 32) * 8
    phases = {k: round(v, 4) for k, v in acc.items()}
    ht_tf = ht_flops / (acc["half_transform_ms"] / 1e3) / 1e12 if acc.get("half_transform_ms") else None
    ex_tf = syrk_flops / (acc["exchange_ms"] / 1e3) / 1e12 if acc.get("exchange_ms") else None
    j_gbs = j_bytes_streamed / (acc["coulomb_ms"] / 1e3) / 1e9 if acc.get("coulomb_ms") else None
    k_ms = acc.get("half_transform_ms", 0.0) + acc.get("exchange_ms", 0.0)
    k_tf = (ht_flops + syrk_flops) / (k_ms / 1e3) / 1e12 if k_ms else None

    if rank != 0:
        if pg:
            pg.destroy_process_group()
        return
    F_gpu = F.cpu().numpy()
    cpu, F_ref = (None, None) if args.no_cpu_baseline else cpu_reference_rate(inp)
    parity = None
    if F_ref is not None:
        parity = dict(max_abs_F_minus_reference=float(np.abs(F_gpu - F_ref).max()), tolerance=1e-10,
                      reference="nonRelFockMatrix compiled from the reference's sources, on the timed build's inputs")
    del dev, src, store
    torch.cuda.empty_cache()
    scf_block = scf_times(torch, want_cpu=not args.no_cpu_baseline)
    rkb_block = rkb_fock_times(torch, fp64_peak, want_cpu=not args.no_cpu_baseline)
    mo_block = mo_transform_block(torch, fp64_peak, want_cpu=not args.no_cpu_baseline)
    orb_block = orbital_optimization_block()
    x2c_block = x2c_batch_block(want_cpu=not args.no_cpu_baseline)
    gnof_block = gnof_optimization_block()
    int_block = integrals_block(torch, hbm_peak, want_cpu=not args.no_cpu_baseline)
    rel_block = rel_scf_times(not args.no_cpu_baseline,
                              (rkb_block.get("reference_cpu") or {}).get("seconds_per_build"))
    line = dict(
        metric=METRIC, value=value, unit=UNIT, n_gpus=ws, steps=args.steps, warmup=args.warmup,
        ms_per_step=1e3 * t / args.steps, higher_is_better=True, scaling="weak", vs_baseline=None, dtype="f64",
        data="synthetic",
        config=bench_config(ws),
        roofline={"bound": "tensor", "kernel": HT["kernel"],
                  "achieved": ht_tf, "peak": fp64_peak, "unit": "TFLOP/s",
                  "frac": (ht_tf / fp64_peak) if (ht_tf and fp64_peak) else None, "traffic": HT["traffic"],
                  "traffic_source": ("dram read+write of one launch, ncu capture in " + HT["profile"])
                  if HT["traffic"] else "no ncu capture of this kernel yet",
                  "algorithmic_bytes": 8.0 * N_AUX * (N_AO * N_AO + N_OCC * N_AO),
                  "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (FP64 has no entry in MEASURED_PEAKS.json)",
                  "algorithmic": "2*naux*nocc*n^2 flops per launch (one launch per build)"},
        exchange={"bound": "tensor", "kernel": "half-transform + SYRK (FP64 DMMA)", "achieved": k_tf,
                  "peak": fp64_peak, "unit": "TFLOP/s", "frac": (k_tf / fp64_peak) if (k_tf and fp64_peak) else None,
                  "algorithmic": "2*naux*nocc*n^2 (half-transform) + 2*naux*nocc*15*80*80 (the SYRK's executed "
                                 "upper tiles) flops per build"},
        coulomb={"bound": "hbm", "achieved": j_gbs, "peak": hbm_peak, "unit": "GB/s",
                 "frac": (j_gbs / hbm_peak) if j_gbs else None, "peak_source": hbm_src,
                 "algorithmic": "2*naux*n^2*8 bytes per build (two passes over B)",
                 "streamed": "2*naux*n(n+1)/2*8 bytes: both passes stream the packed upper triangles of the "
                             "symmetric B^P, on a side stream from the top of the build (beside the occupied "
                             "recovery and the half-transform, one CTA per SM); achieved counts the streamed bytes",
                 "algorithmic_rate_gbs": (j_bytes / (acc["coulomb_ms"] / 1e3) / 1e9) if acc.get("coulomb_ms") else None},
        kernels={"half_transform_tflops": ht_tf, "syrk_tflops_executed": ex_tf},
        phases_ms=phases, clocks=clk, e2e=e2e, gpu_launches=int(launches), cpu_baseline=cpu, parity=parity,
        time_to_1e8_ha=scf_block,
        time_to_1e8_ha_relativistic=rel_block,
        rkb_fock_4c=rkb_block,
        mo_transform=mo_block,
        orbital_optimization=orb_block,
        x2c_batch=x2c_block,
        gnof_optimization=gnof_block,
        integrals=int_block,
    )
    print(json.dumps(line))
    if pg:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
