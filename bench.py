"""Benchmark: bit-exact negacyclic products/s at N=32768 with an 868-bit q.

One JSON line on rank 0 (contract of the driver):
  value      products/s over all ranks with inputs resident in HBM (a step is one
             pass over a batch of independent products), device-timed;
  e2e        the same metric through the C ABI's host-buffer batch call
             (pm_multiply_host_batch) from pinned host memory: H2D of a, b and
             D2H of c inside the timed region;
  roofline   the dominant kernel's algorithmic bytes per launch / its mean
             device time (CUDA events on its launch stream, recorded by the
             library during the timed steps);
  cpu_baseline  the reference's own rns kernels run by its CPU emulation
             (oracle/_ref/rns_emulated, one product per host core at once) on a
             bounded sample of the same workload; the C restatement of the
             method (oracle/, all host threads) beside it.

Multi-GPU is replicas only: the method has no exchange step between products,
so each rank runs its own batch and value sums products over the max-over-
ranks device time.

--impl reference times the reference's CPU path on the host cores: its own
rns kernel bodies under its CPU emulation (its GPU path needs the closed cuPQC
SDK), one single-threaded process per core, a step being one product at the
same N and width (q = 2^868 - 11993087: the only form that backend takes).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "fherma-polymul-baseline_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "bit-exact products/s at N=32768, 868-bit q"
UNIT = "products/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ring", type=int, default=32768, help="ring dimension N")
    ap.add_argument("--bits", type=int, default=868)
    ap.add_argument("--batch", type=int, default=512, help="independent products per step")
    ap.add_argument("--e2e-batch", type=int, default=0,
                    help="products per step of the end-to-end (host buffer) measurement; 0: the same as "
                         "--batch on one GPU, 64 per rank on several")
    ap.add_argument("--path", default="tensor", choices=["tensor", "simt"],
                    help="tensor: tcgen05 INT8 conversion/CRT (default); simt: the plain CUDA-core method")
    ap.add_argument("--seed", type=int, default=20261203)
    ap.add_argument("--cpu-seconds", type=float, default=5.0,
                    help="seconds of the C restatement's sample (0 skips every CPU baseline)")
    ap.add_argument("--serve-requests", type=int, default=10000,
                    help="requests in the serving stream (0 skips it)")
    ap.add_argument("--serve-rate", type=float, default=6000.0, help="Poisson arrival rate, requests/s")
    ap.add_argument("--uneven", type=int, default=64, help="products in the uneven batch (0 skips it)")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="keep the default launch shapes instead of the autotuner's")
    ap.add_argument("--group", type=int, default=0,
                    help="products per launch group (default launch shapes otherwise; skips the autotuner)")
    ap.add_argument("--conversion", choices=["whole", "groups"], default="whole",
                    help="tensor path conversion for --ncu-case: whole (K1W, the whole basis per tile, "
                         "the default) or groups (K1T, one group of 16 primes per tile)")
    ap.add_argument("--ncu-case", type=int, default=0, metavar="K",
                    help="no timing: one batched call of K products in one launch group (one launch per pass), "
                         "for an ncu capture")
    return ap.parse_args()


def seeded_q(seed, bits):
    import numpy as np

    rng = np.random.default_rng(seed)
    q = 0
    for _ in range((bits + 31) // 32):
        q = (q << 32) | int(rng.integers(0, 2**32))
    q &= (1 << bits) - 1
    return q | (1 << (bits - 1)) | 1


# ---------------------------------------------------------------------------
# distributed plumbing (replicas)
# ---------------------------------------------------------------------------
def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def max_over_ranks(value, dist, world, device):
    """The slowest rank's time: every rank contributes, every rank gets the max."""
    if world <= 1:
        return value
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def init_dist(world, backend):
    import datetime

    import torch.distributed as dist

    if world > 1 and not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return dist


# ---------------------------------------------------------------------------
# CPU arms
# ---------------------------------------------------------------------------
def cpu_sample(a, b, q, seconds, threads):
    """Run the oracle port on (a, b) repeatedly for ~seconds; return products/s and count."""
    from oracle import oracle

    oracle.rns_multiply(a[:64], b[:64], q, threads=threads)  # load + warm
    done, t0 = 0, time.perf_counter()
    while True:
        oracle.rns_multiply(a, b, q, threads=threads)
        done += 1
        el = time.perf_counter() - t0
        if el >= seconds:
            return done / el, done, el


def host_inputs(n, q, seed, count=1):
    import numpy as np

    from tests.helpers import uniform_below

    rng = np.random.default_rng(seed)
    limbs = (q.bit_length() + 63) // 64
    return [(uniform_below(rng, q, n, limbs), uniform_below(rng, q, n, limbs)) for _ in range(count)]


FHERMA_Q = (1 << 868) - 11993087  # the reference's point: its rns backend takes only q = 2^868 - c, c < 2^28


def emulated_reference_sample(n, products, workers, seed):
    """The reference's own rns kernels, CPU-emulated (oracle/_ref/rns_emulated): `products`
    products at (n, 2^868 - 11993087) split over `workers` concurrent processes (the
    emulation runs one host thread each).  Returns (products/s over the wall time of the
    whole sample, wall seconds, per-case seconds, one (a, b, c) triple to check)."""
    import tempfile

    import numpy as np

    from tests import reference_emulation as emu
    from tests.helpers import uniform_below

    rng = np.random.default_rng(seed)
    pairs = [(uniform_below(rng, FHERMA_Q, n, 14), uniform_below(rng, FHERMA_Q, n, 14)) for _ in range(products)]
    workers = max(1, min(workers, products))
    parts = [pairs[w::workers] for w in range(workers)]
    with tempfile.TemporaryDirectory() as tmp:
        dirs = []
        for w, part in enumerate(parts):
            d = os.path.join(tmp, f"w{w}")
            emu.write_point(d, n, FHERMA_Q, part)
            dirs.append(d)
        t0 = time.perf_counter()
        procs = [emu.start(d) for d in dirs]
        for p in procs:
            _, err = p.communicate()
            if p.returncode != 0:
                raise RuntimeError(f"emulated reference failed: {err[-300:]}")
        wall = time.perf_counter() - t0
        secs = []
        outs0 = None
        for w, (d, part) in enumerate(zip(dirs, parts)):
            outs, sec = emu.read_results(d, len(part), n)
            secs += sec
            if w == 0:
                outs0 = outs[0]
    a, b = parts[0][0]
    return products / wall, wall, secs, (a, b, outs0)


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def run_reference(args):
    """The reference's CPU path on the host cores: its own rns kernel bodies run by its CPU
    emulation (oracle/_ref/rns_emulated, one host thread per process), one process per core;
    a step is one product at the bench's N.  Falls back to the oracle's C restatement of the
    method (threads over primes) when the emulated binary was not built."""
    world, rank, _ = dist_env()
    if rank != 0:
        return
    from tests import reference_emulation as emu

    cores = host_cores()
    base = {
        "impl": "reference", "metric": METRIC, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic",
    }
    if emu.available():
        import numpy as np

        from oracle import oracle

        # warm-up: the binary, libgmp and the page cache, on small rings
        emulated_reference_sample(1024, max(1, min(args.warmup, cores)), cores, args.seed + 2)
        value, wall, secs, (a, b, c) = emulated_reference_sample(args.ring, args.steps, cores, args.seed + 1)
        if not (c == oracle.rns_multiply(a, b, FHERMA_Q)).all():
            raise SystemExit("emulated reference disagrees with the oracle")
        per = sorted(secs)
        line = dict(base, value=value, ms_per_step=1000 * wall / args.steps)
        line["config"] = {"workload": f"one negacyclic product per step, N={args.ring}, 868-bit q = 2^868 - 11993087 "
                                      "(the reference's rns backend takes only q = 2^868 - c), coefficients uniform "
                                      "in [0, q)", "n": args.ring, "q_bits": 868,
                          "parallelism": f"{min(cores, args.steps)} concurrent single-threaded processes"}
        line["cpu_baseline"] = {"value": value, "unit": UNIT, "cores": min(cores, args.steps), "kind": "reference",
                                "sample": f"{args.steps} products at N={args.ring} through the reference's own rns "
                                          "kernels (rns/solve.cu) run by its CPU emulation (tests/build_emulation.py "
                                          "rewrite, GMP big integers), one process per core; "
                                          f"{per[len(per) // 2]:.1f} s per product (median)",
                                "seconds_per_product_median": per[len(per) // 2]}
        line["e2e"] = {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
        print(json.dumps(line), flush=True)
        return

    threads = os.cpu_count() or 1
    q = seeded_q(args.seed, args.bits)
    (a, b), = host_inputs(args.ring, q, args.seed + 1)
    from oracle import oracle

    for _ in range(max(args.warmup, 1)):
        oracle.rns_multiply(a, b, q, threads=threads)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        oracle.rns_multiply(a, b, q, threads=threads)
    el = time.perf_counter() - t0
    value = args.steps / el
    line = dict(base, value=value, ms_per_step=1000 * el / args.steps)
    line["config"] = {"workload": f"one negacyclic product per step, N={args.ring}, {args.bits}-bit seeded odd q, "
                                  "coefficients uniform in [0, q)", "n": args.ring, "q_bits": args.bits,
                      "parallelism": "cpu threads"}
    line["cpu_baseline"] = {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                            "sample": f"{args.steps} products at N={args.ring}; the reference's RNS method restated "
                                      "in C (oracle/polymul_oracle.c), threads over primes (the emulated reference "
                                      "binary was not built)"}
    line["e2e"] = {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_uuid):
        self.uuid = device_uuid
        self.proc = None
        self.lines = []

    def start(self):
        cmd = ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits", "-lms", "50"]
        if self.uuid:
            cmd += ["-i", self.uuid]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=5)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for name, flag in zip(names, f[5:9]):
                if flag.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def device_inputs(torch, batch, n, limbs, q, seed):
    """Seeded coefficients uniform in [0, q) generated on the device by rejection."""
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    bits = q.bit_length()
    top = bits - 64 * (limbs - 1)
    q_limbs = [(q >> (64 * j)) & ((1 << 64) - 1) for j in range(limbs)]
    sign = -(1 << 63)

    def order_key(v):  # an unsigned limb as the int64 that sorts the same way
        s = v ^ (1 << 63)
        return s - (1 << 64) if s >= (1 << 63) else s

    q_s = torch.tensor([order_key(v) for v in q_limbs], dtype=torch.int64, device="cuda")

    def draw(rows):
        hi = torch.randint(0, 2**32, (rows, n, limbs), dtype=torch.int64, device="cuda", generator=g)
        lo = torch.randint(0, 2**32, (rows, n, limbs), dtype=torch.int64, device="cuda", generator=g)
        x = (hi << 32) | lo
        x[..., limbs - 1] &= (1 << top) - 1 if top < 64 else -1
        return x

    out = draw(batch)
    for _ in range(64):
        xs = out ^ sign  # unsigned order as signed order
        less = torch.zeros(out.shape[:2], dtype=torch.bool, device="cuda")
        equal = torch.ones_like(less)
        for j in range(limbs - 1, -1, -1):
            less |= equal & (xs[..., j] < q_s[j])
            equal &= xs[..., j] == q_s[j]
        bad = ~less
        nbad = int(bad.sum())
        if nbad == 0:
            return out
        fresh = draw(1).reshape(n, limbs)
        while fresh.shape[0] < nbad:
            fresh = torch.cat([fresh, draw(1).reshape(n, limbs)])
        out[bad] = fresh[:nbad]
    raise RuntimeError("rejection sampling did not converge")


def run_plain(args, torch, plan, A, Bv, Cv, stream, batched_value):
    """The plain single-product path on the same GPU: one product per call.

    device: pm_multiply on device buffers, one launch sequence per product, CUDA-event timed;
    host:   pm_multiply_host on pinned host buffers (the fherma_run call), wall-clock timed."""
    K = min(64, A.shape[0])
    sh = stream.cuda_stream

    def dev_pass():
        for k in range(K):
            plan.multiply(A[k].data_ptr(), Bv[k].data_ptr(), Cv[k].data_ptr(), stream=sh)

    for _ in range(max(args.warmup, 1)):
        dev_pass()
    stream.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        dev_pass()
    e1.record(stream)
    e1.synchronize()
    dev = K * args.steps / (e0.elapsed_time(e1) / 1000.0)

    H = min(8, K)
    ha = A[:H].cpu().pin_memory()
    hb = Bv[:H].cpu().pin_memory()
    hc = torch.empty_like(ha).pin_memory()
    for k in range(H):
        plan.multiply_host_ptr(ha[k].data_ptr(), hb[k].data_ptr(), hc[k].data_ptr())
    t0 = time.perf_counter()
    reps = max(args.steps // 2, 2)
    for _ in range(reps):
        for k in range(H):
            plan.multiply_host_ptr(ha[k].data_ptr(), hb[k].data_ptr(), hc[k].data_ptr())
    host = H * reps / (time.perf_counter() - t0)

    # the plain method too: the same single-product calls with the SIMT conversion and CRT
    import polymul
    simt = polymul.Plan(plan.n, plan.q, coef_limbs=plan.coef_limbs, tensor=False)
    for k in range(min(8, K)):
        simt.multiply(A[k].data_ptr(), Bv[k].data_ptr(), Cv[k].data_ptr(), stream=sh)
    stream.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        for k in range(K):
            simt.multiply(A[k].data_ptr(), Bv[k].data_ptr(), Cv[k].data_ptr(), stream=sh)
    e1.record(stream)
    e1.synchronize()
    simt_dev = K * args.steps / (e0.elapsed_time(e1) / 1000.0)
    simt.close()
    return {"device_products_per_s": dev, "host_products_per_s": host,
            "simt_method_device_products_per_s": simt_dev,
            "batched_over_plain_device": batched_value / dev,
            "api": "pm_multiply (device buffers) and pm_multiply_host (pinned host buffers), one product per call; "
                   "simt_method: PM_CONVERT_SIMT plan, pm_multiply per product",
            "products": {"device": K * args.steps, "host": H * reps}}


def run_fherma_drop_in(args, q, cases=24):
    """The drop-in call itself: fherma_run on the harness's own std::vector inputs (pageable
    memory), timed by the harness around each call, as the reference's published number is.
    Two harnesses run the same point directory of `cases` products at the bench's N and q:
    this repository's runner (polymul_solution) and the reference's unmodified main.cpp linked
    against libfherma_polymul.so (oracle/_ref/fherma_main, when it was built).  Per-case
    seconds come from their results.json; c.bin files are checked against the oracle on two
    cases."""
    import tempfile

    import numpy as np

    from oracle import oracle
    from tests import reference_emulation as emu

    n, limbs = args.ring, (args.bits + 63) // 64
    if limbs != 14:
        return None
    harnesses = {"polymul_solution": os.path.join(PKG, "polymul_solution"),
                 "reference_main_cpp": os.path.join(ROOT, "oracle", "_ref", "fherma_main")}
    rng = np.random.default_rng(args.seed + 97)
    from tests.helpers import uniform_below

    pairs = [(uniform_below(rng, q, n, 14), uniform_below(rng, q, n, 14)) for _ in range(4)]
    out = {"cases": cases, "n": n, "api": "fherma_run (fherma.h:45) on std::vector inputs, harness-timed"}
    with tempfile.TemporaryDirectory() as tmp:
        # the point directory format the reference's harness reads (main.cpp:137-208); 4 distinct
        # input pairs cycled over the cases
        emu.write_point(tmp, n, q, [pairs[k % len(pairs)] for k in range(cases)])
        for name, exe in harnesses.items():
            if not os.path.exists(exe):
                continue
            res_dir = os.path.join(tmp, "out")
            r = subprocess.run([exe, tmp], capture_output=True, text=True, timeout=600)
            if r.returncode != 0:
                out[name] = {"error": r.stderr[-300:]}
                continue
            got, secs = emu.read_results(tmp, cases, n)
            for k in (0, 1):
                a, b = pairs[k]
                if not (got[k] == oracle.rns_multiply(a, b, q)).all():
                    raise SystemExit(f"{name}: fherma_run output differs from the oracle")
            us = sorted(1e6 * x for x in secs[1:])  # the first call pays one-time staging set-up
            pick = lambda f: us[min(len(us) - 1, int(f * (len(us) - 1) + 0.5))]  # noqa: E731
            out[name] = {"p50_us": pick(0.5), "p99_us": pick(0.99), "min_us": us[0], "mean_us": sum(us) / len(us),
                         "first_call_us": 1e6 * secs[0]}
            import shutil

            shutil.rmtree(res_dir, ignore_errors=True)
    return out


def run_special(args, torch, polymul, tuning):
    """The reference's FHERMA modulus q = 2^868 - 11993087, a special-form prime: device products/s
    with the folding reduction (PM_SPECIAL_FORM) and with the general one (the default), same
    batch and launch shapes, bit-identical results checked; and through the direct wide-modulus
    NTT (PM_WIDE_NTT), the reference's wide backend, for comparison."""
    import numpy as np

    n, limbs = args.ring, 14
    q = (1 << 868) - 11993087
    B = min(args.batch, 256)
    A = device_inputs(torch, B, n, limbs, q, args.seed + 71)
    Bv = device_inputs(torch, B, n, limbs, q, args.seed + 73)
    out = {"q": "2^868 - 11993087", "batch": B}
    results = []
    for label, special in (("special_form", True), ("general_reduction", False)):
        plan = polymul.Plan(n, q, coef_limbs=limbs, tensor=(args.path == "tensor"), special_form=special)
        if tuning and "row_radix" in tuning:
            plan.set_tuning(tuning["row_radix"], tuning["conv_ctas_per_sm"], tuning["crt_ctas_per_sm"],
                            tuning["group"], tuning["row_persistent"], tuning["conv_whole_basis"])
        elif args.group:
            plan.set_tuning(group=args.group)
        C = torch.empty_like(A)
        st = torch.cuda.Stream()
        for _ in range(max(args.warmup, 1)):
            plan.multiply_batch(A.data_ptr(), Bv.data_ptr(), C.data_ptr(), B, stream=st.cuda_stream)
        st.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(args.steps):
            plan.multiply_batch(A.data_ptr(), Bv.data_ptr(), C.data_ptr(), B, stream=st.cuda_stream)
        e1.record(st)
        e1.synchronize()
        out[label + "_products_per_s"] = B * args.steps / (e0.elapsed_time(e1) / 1000.0)
        results.append(C[:4].cpu().numpy().view(np.uint64))
        plan.close()
    out["identical"] = bool(all((results[0] == results[1]).flatten()))
    out["speedup"] = out["special_form_products_per_s"] / out["general_reduction_products_per_s"]
    # the reference's quartic factorization (PM_QUARTIC) on the same batch: 16 primes x 4 channels
    try:
        quart = polymul.Plan(n, q, coef_limbs=limbs, quartic=True)
        C = torch.empty_like(A)
        st = torch.cuda.Stream()
        for _ in range(max(args.warmup, 1)):
            quart.multiply_batch(A.data_ptr(), Bv.data_ptr(), C.data_ptr(), B, stream=st.cuda_stream)
        st.synchronize()
        polymul.profile_enable(3 * B * args.steps + 16)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(args.steps):
            quart.multiply_batch(A.data_ptr(), Bv.data_ptr(), C.data_ptr(), B, stream=st.cuda_stream)
        e1.record(st)
        e1.synchronize()
        prof = polymul.profile_read()
        polymul.profile_enable(0)
        out["quartic_products_per_s"] = B * args.steps / (e0.elapsed_time(e1) / 1000.0)
        out["quartic_us_per_product"] = {k: 1000.0 * v[1] / (B * args.steps) for k, v in prof.items()}
        out["quartic_identical"] = bool((C[:4].cpu().numpy().view(np.uint64) == results[1]).all())
        out["quartic_over_general"] = out["quartic_products_per_s"] / out["general_reduction_products_per_s"]
        quart.close()
    except polymul.PolymulError as e:
        out["quartic"] = f"not applicable at n={n}: {e}"
    # the direct wide-modulus NTT (PM_WIDE_NTT) on the same prime, for comparison: 64 products
    Bw = min(B, 64)
    try:
        wide = polymul.Plan(n, q, coef_limbs=limbs, wide=True)
    except polymul.PolymulError as e:  # this prime is 1 mod 2n only up to n = 32768
        out["wide_ntt"] = f"not applicable at n={n}: {e}"
        del A, Bv
        torch.cuda.empty_cache()
        return out
    Cw = torch.empty_like(A[:Bw])
    st = torch.cuda.Stream()
    wide.multiply_batch(A.data_ptr(), Bv.data_ptr(), Cw.data_ptr(), Bw, stream=st.cuda_stream)
    st.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(max(args.steps // 2, 1)):
        wide.multiply_batch(A.data_ptr(), Bv.data_ptr(), Cw.data_ptr(), Bw, stream=st.cuda_stream)
    e1.record(st)
    e1.synchronize()
    out["wide_ntt_products_per_s"] = Bw * max(args.steps // 2, 1) / (e0.elapsed_time(e1) / 1000.0)
    out["wide_ntt_identical"] = bool((Cw[:4].cpu().numpy().view(np.uint64) == results[1]).all())
    out["rns_over_wide"] = out["general_reduction_products_per_s"] / out["wide_ntt_products_per_s"]
    wide.close()
    del A, Bv
    torch.cuda.empty_cache()
    return out


def run_uneven(args, torch, polymul):
    """64 products, N log-uniform over {1024..65536}, widths uniform in 200..868 bits
    (seed 4), as one autotuned graph; against the same products through per-product
    plans, one launch sequence after another on one stream."""
    import numpy as np

    from tests.helpers import uniform_below

    rng = np.random.default_rng(4)
    K = args.uneven
    ns = [1024 << int(k) for k in rng.integers(0, 7, size=K)]
    widths = [int(w) for w in rng.integers(200, 869, size=K)]
    qs = []
    for w in widths:
        q = int(rng.integers(0, 2**62)) | 1
        while q.bit_length() < w:
            q = (q << 62) | int(rng.integers(0, 2**62))
        qs.append((q & ((1 << w) - 1)) | (1 << (w - 1)) | 1)
    a = [uniform_below(rng, q, n, 14) for q, n in zip(qs, ns)]
    b = [uniform_below(rng, q, n, 14) for q, n in zip(qs, ns)]
    batch = polymul.Batch(ns, qs, coef_limbs=14)
    pa, pb = batch.pack(a), batch.pack(b)
    batch.copy_in(pa.ctypes.data, pb.ctypes.data)
    torch.cuda.synchronize()
    tuned_us = batch.autotune(reps=3)
    st = torch.cuda.Stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    batch.run(st.cuda_stream)
    reps = 5
    e0.record(st)
    for _ in range(reps):
        batch.run(st.cuda_stream)
    e1.record(st)
    e1.synchronize()
    batch_us = 1000.0 * e0.elapsed_time(e1) / reps
    batch.check_errors()
    pc = np.zeros_like(pa)
    batch.copy_out(pc.ctypes.data)
    torch.cuda.synchronize()
    got = batch.unpack(pc)
    # the same products through per-product plans (tensor path), sequentially on one stream
    plans = [polymul.Plan(n, q, 14, tensor=True) for n, q in zip(ns, qs)]
    da = [torch.from_numpy(x.view(np.int64)).cuda() for x in a]
    db = [torch.from_numpy(x.view(np.int64)).cuda() for x in b]
    dc = [torch.empty_like(x) for x in da]
    for p, x, y, z in zip(plans, da, db, dc):
        p.multiply(x.data_ptr(), y.data_ptr(), z.data_ptr(), 0, st.cuda_stream)
    e0.record(st)
    for _ in range(reps):
        for p, x, y, z in zip(plans, da, db, dc):
            p.multiply(x.data_ptr(), y.data_ptr(), z.data_ptr(), 0, st.cuda_stream)
    e1.record(st)
    e1.synchronize()
    seq_us = 1000.0 * e0.elapsed_time(e1) / reps
    mismatches = sum(int((dc[z].cpu().numpy().view(np.uint64) != got[z]).any(axis=1).sum()) for z in range(K))
    for p in plans:
        p.close()
    batch.close()
    return {"workload": f"{K} products, N log-uniform over 1024..65536, q widths uniform in 200..868 bits (seed 4)",
            "us_per_batch": batch_us, "products_per_s": K / (batch_us * 1e-6), "autotuned_us": tuned_us,
            "per_product_plans_us": seq_us, "per_product_plans_products_per_s": K / (seq_us * 1e-6),
            "coefficients": int(sum(ns)), "mismatches_vs_per_product_plans": mismatches}


SERVE_SIZES = (4096, 16384, 32768, 65536)
SERVE_WEIGHTS = (0.4, 0.3, 0.2, 0.1)


def run_serving(args, torch, polymul):
    """Poisson arrivals of products of mixed N (868-bit q) through the serving loop,
    and the same arrival schedule through the plain path one request at a time."""
    import numpy as np

    rng = np.random.default_rng(5)
    R = args.serve_requests
    q = seeded_q(args.seed + 5, args.bits)
    limbs = (args.bits + 63) // 64
    sizes = rng.choice(SERVE_SIZES, size=R, p=SERVE_WEIGHTS)
    arrivals = np.cumsum(rng.exponential(1.0 / args.serve_rate, size=R))
    pool_k, ring = 4, 32  # distinct inputs per size; output buffers per size (reused round robin)
    pools = {}
    for n in SERVE_SIZES:
        a = device_inputs(torch, pool_k, n, limbs, q, args.seed + n).cpu().pin_memory()
        b = device_inputs(torch, pool_k, n, limbs, q, args.seed + 3 * n).cpu().pin_memory()
        c = torch.zeros((ring, n, limbs), dtype=torch.int64).pin_memory()
        pools[n] = (a, b, c)
    last_input = {}  # (n, ring slot) -> input index of the last request written there

    def run(submit, drain, arr=arrivals, count_to=R):
        count = {n: 0 for n in SERVE_SIZES}
        t0 = time.perf_counter()
        for k in range(count_to):
            n = int(sizes[k])
            j, r = count[n] % pool_k, count[n] % ring
            count[n] += 1
            while time.perf_counter() - t0 < arr[k]:
                pass
            a, b, c = pools[n]
            submit(n, a[j].data_ptr(), b[j].data_ptr(), c[r].data_ptr(), t0 + arr[k])
            last_input[(n, r)] = j
        drain()
        return time.perf_counter() - t0

    # the serving loop
    srv = polymul.Server(slots=8, max_group=4, tensor=(args.path == "tensor"))
    for n in SERVE_SIZES:  # plans (tables) resident before the stream starts
        a, b, c = pools[n]
        srv.wait(srv.submit_ptr(n, q, limbs, a[0].data_ptr(), b[0].data_ptr(), c[0].data_ptr()))
    srv.reset_stats()
    wall = run(lambda n, pa, pb, pc, due: srv.submit_ptr(n, q, limbs, pa, pb, pc), srv.drain)
    st = srv.stats()
    # saturation: the same mix queued all at once, what the loop sustains when the link is the limit
    srv.reset_stats()
    S = min(R, 4000)
    sat_wall = run(lambda n, pa, pb, pc, due: srv.submit_ptr(n, q, limbs, pa, pb, pc), srv.drain,
                   np.zeros(S), S)
    sat = srv.stats()
    srv.close()
    mismatches = 0
    plans = {n: polymul.Plan(n, q, limbs) for n in SERVE_SIZES}
    for (n, r), j in last_input.items():
        if r >= 2:
            continue
        a, b, c = pools[n]
        want = plans[n].multiply_host(a[j].numpy().view(np.uint64), b[j].numpy().view(np.uint64))
        mismatches += int((c[r].numpy().view(np.uint64) != want).any(axis=1).sum())

    # the plain path in turn: one pm_multiply_host at a time, same arrival schedule
    lat = []

    def plain_submit(n, pa, pb, pc, due):
        polymul.check(polymul.lib().pm_multiply_host(plans[n].handle, pa, pb, pc))
        lat.append((time.perf_counter() - due) * 1e6)

    plain_wall = run(plain_submit, lambda: None)
    for p in plans.values():
        p.close()
    lat.sort()
    pct = lambda v, f: v[min(len(v) - 1, int(f * (len(v) - 1) + 0.5))]  # noqa: E731
    return {
        "workload": f"{R} requests, Poisson arrivals at {args.serve_rate:.0f}/s (seed 5), N in {SERVE_SIZES} "
                    f"with weights {SERVE_WEIGHTS}, {args.bits}-bit q, pinned host buffers",
        "products_per_s": st["products_per_s"], "p50_us": st["p50_us"], "p99_us": st["p99_us"],
        "mean_us": st["mean_us"], "wall_s": wall, "groups": st["groups"], "peak_inflight": st["peak_inflight"],
        "peak_group": st["peak_group"], "mismatches": mismatches,
        "saturated": {"requests": S, "products_per_s": S / sat_wall, "p50_us": sat["p50_us"], "p99_us": sat["p99_us"],
                      "peak_inflight": sat["peak_inflight"], "peak_group": sat["peak_group"],
                      "note": "all requests queued at t=0: latency is queueing time"},
        "plain_in_turn": {"products_per_s": R / plain_wall, "p50_us": pct(lat, 0.5), "p99_us": pct(lat, 0.99),
                          "api": "pm_multiply_host, one request at a time"},
    }


def algorithmic_bytes(n, primes, limbs):
    """Mandatory HBM bytes of each kernel per product: inputs read once, residue
    planes written and read once, output written once (twiddle and table reads are
    implementation overhead and not counted)."""
    io = n * 8 * limbs
    conv = 2 * io + 2 * primes * n * 4
    rows = 2 * primes * n * 4 + primes * n * 4
    crt = primes * n * 4 + io
    return {"k1_convert_cols": conv, "k1t_convert_cols": conv, "k2_rows": rows,
            "k3_cols_crt": crt, "k3t_cols_crt": crt}


def pcie_bandwidth(torch, device, nbytes=256 << 20, reps=4):
    """Pinned host <-> device copy rates (GB/s), each direction alone, CUDA events on a side stream."""
    h = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    d = torch.empty(nbytes, dtype=torch.uint8, device=f"cuda:{device}")
    st = torch.cuda.Stream()
    out = {}
    for name, dst, src in (("h2d_gbs", d, h), ("d2h_gbs", h, d)):
        with torch.cuda.stream(st):
            dst.copy_(src, non_blocking=True)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            for _ in range(reps):
                dst.copy_(src, non_blocking=True)
            e1.record(st)
        e1.synchronize()
        out[name] = reps * nbytes / (e0.elapsed_time(e1) / 1000.0) / 1e9
    # both directions at once (what the host-buffer pipeline does): H2D of a pinned buffer on
    # one stream while a D2H of half that size runs on another, as for a, b in and c out
    h2 = torch.empty(nbytes // 2, dtype=torch.uint8, pin_memory=True)
    d2 = torch.empty(nbytes // 2, dtype=torch.uint8, device=f"cuda:{device}")
    st2 = torch.cuda.Stream()
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    ev[0].record(st)
    ev[2].record(st2)
    st2.wait_event(ev[0])
    with torch.cuda.stream(st):
        for _ in range(reps):
            d.copy_(h, non_blocking=True)
    with torch.cuda.stream(st2):
        for _ in range(reps):
            h2.copy_(d2, non_blocking=True)
    ev[1].record(st)
    ev[3].record(st2)
    torch.cuda.synchronize()
    out["h2d_gbs_with_d2h"] = reps * nbytes / (ev[0].elapsed_time(ev[1]) / 1000.0) / 1e9
    out["d2h_gbs_with_h2d"] = reps * (nbytes // 2) / (ev[0].elapsed_time(ev[3]) / 1000.0) / 1e9
    del h, d, h2, d2
    return out


def run_ours(args):
    import numpy as np
    import torch

    import polymul

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    dist = init_dist(world, "nccl")
    n, bits = args.ring, args.bits
    q = seeded_q(args.seed, bits)
    limbs = (bits + 63) // 64
    plan = polymul.Plan(n, q, coef_limbs=limbs, tensor=(args.path == "tensor"))
    tuning = None
    if args.group:
        plan.set_tuning(group=args.group)
        tuning = {"group": args.group, "source": "--group"}
    elif args.autotune:
        tuning = plan.autotune(reps=8)
    B = args.batch
    A = device_inputs(torch, B, n, limbs, q, args.seed + 17 + 1000 * rank)
    Bv = device_inputs(torch, B, n, limbs, q, args.seed + 29 + 1000 * rank)
    Cv = torch.empty_like(A)
    stream = torch.cuda.Stream()
    sh = stream.cuda_stream

    def step():
        plan.multiply_batch(A.data_ptr(), Bv.data_ptr(), Cv.data_ptr(), B, stream=sh)

    # bit-exact check of sampled products against the oracle (outside the timed region)
    from oracle import oracle

    step()
    stream.synchronize()
    mismatches, checked = 0, 0
    for k in sorted({0, B // 2, B - 1}):
        a = A[k].cpu().numpy().view(np.uint64)
        b = Bv[k].cpu().numpy().view(np.uint64)
        c = Cv[k].cpu().numpy().view(np.uint64)
        mismatches += int((oracle.rns_multiply(a, b, q) != c).any(axis=1).sum())
        checked += 1
    if mismatches:
        raise SystemExit(f"bench aborted: {mismatches} mismatching coefficients against the oracle")

    for _ in range(max(args.warmup - 1, 0)):
        step()
    stream.synchronize()
    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(local).uuid)
    except Exception:
        pass
    sampler = ClockSampler(uuid)

    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    polymul.profile_enable(3 * B * args.steps + 16)
    launches0 = polymul.launch_count()
    sampler.start()
    time.sleep(0.1)  # let the sampler attach before the timed region
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        step()
    ev1.record(stream)
    ev1.synchronize()
    clocks = sampler.stop()
    launches = polymul.launch_count() - launches0
    prof = polymul.profile_read()
    polymul.profile_enable(0)
    ms = max_over_ranks(ev0.elapsed_time(ev1), dist, world, "cuda")
    total_products = B * args.steps * world
    value = total_products / (ms / 1000.0)

    plain = run_plain(args, torch, plan, A, Bv, Cv, stream, value / world)
    if world == 1:
        plain["fherma_run"] = run_fherma_drop_in(args, q)

    # end to end through the C ABI host-buffer call, pinned host memory
    # the whole batch on one GPU; 64 products a rank when several ranks share the host's pinned memory
    E = min(args.e2e_batch or (B if world == 1 else 64), B)
    ha = torch.empty((E, n, limbs), dtype=torch.int64, pin_memory=True)
    hb = torch.empty_like(ha, pin_memory=True)
    hc = torch.empty_like(ha, pin_memory=True)
    ha.copy_(A[:E])
    hb.copy_(Bv[:E])
    del A, Bv, Cv
    torch.cuda.empty_cache()
    def e2e_step():
        plan.multiply_host_batch_ptr(ha.data_ptr(), hb.data_ptr(), hc.data_ptr(), E)

    for _ in range(max(args.warmup, 1)):
        e2e_step()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0, dist, world, "cuda")
    e2e_value = E * args.steps * world / e2e_s
    io = n * 8 * limbs
    link = pcie_bandwidth(torch, local)
    # the copies bound the host-buffer call: 2 polynomials in and 1 out per product, the two
    # directions on separate copy engines at the rates measured while both run
    link["bound_products_per_s"] = 1.0 / max(2 * io / (link["h2d_gbs_with_d2h"] * 1e9),
                                             io / (link["d2h_gbs_with_h2d"] * 1e9))
    link["bound_one_direction_at_a_time"] = 1.0 / max(2 * io / (link["h2d_gbs"] * 1e9), io / (link["d2h_gbs"] * 1e9))
    link["frac"] = e2e_value / world / link["bound_products_per_s"]

    # roofline of the dominant kernel
    alg = algorithmic_bytes(n, plan.primes, limbs)
    dom = max(prof, key=lambda k: prof[k][1]) if prof else None
    roofline = None
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak, peak_src = 6650.0, "fallback"
    if os.path.exists(peaks_path):
        peak = float(json.load(open(peaks_path))["hbm_gbs"])
        peak_src = "measured"
    # each launch covers a group of products; bytes per launch = per-product bytes x products per launch
    timed_products = B * args.steps
    kernels = {}
    total_ms = sum(v[1] for v in prof.values()) or 1.0
    for name, (cnt, tot) in prof.items():
        per_launch = alg.get(name, 0) * timed_products / cnt
        kernels[name] = {"launches": cnt, "mean_us": 1000 * tot / cnt, "share": tot / total_ms,
                         "products_per_launch": timed_products / cnt,
                         "achieved_gbs": per_launch / (tot / cnt / 1000.0) / 1e9 if name in alg else None}
    if dom:
        cnt, tot = prof[dom]
        per_launch = alg[dom] * timed_products / cnt
        achieved = per_launch / (tot / cnt / 1000.0) / 1e9
        # DRAM bytes come from ncu captures only (a profiler run is never a timed run): not measured here
        roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                    "frac": achieved / peak, "peak_source": peak_src,
                    "traffic": None,
                    "algorithmic_bytes_per_launch": per_launch,
                    "algorithmic_bytes_per_product": alg[dom]}

    # INT8 tensor-core contractions (tensor path): algorithmic INT8 ops per product over each
    # kernel's device time, against the INT8 dense peak taken as twice the measured bf16 GEMM rate
    # (B200: 4.5 vs 2.25 PFLOP/s nominal); the MMAs issue more (K padded to 128 and 256 bytes)
    tensor_pipe = None
    if args.path == "tensor":
        digits = (bits + 7) // 8
        ops = {"k1t_convert_cols": 2 * (2 * n) * digits * 4 * plan.primes,
               "k3t_cols_crt": 2 * n * 4 * plan.primes * (digits + 3)}
        bf16 = 1590.0
        if os.path.exists(peaks_path):
            bf16 = float(json.load(open(peaks_path)).get("bf16_tflops", bf16))
        tensor_pipe = {}
        for name, per in ops.items():
            if name in prof:
                cnt, tot = prof[name]
                tops = per * timed_products / (tot / 1000.0) / 1e12
                tensor_pipe[name] = {"int8_ops_per_product": per, "achieved_tops": tops,
                                     "peak_tops": 2 * bf16, "frac": tops / (2 * bf16),
                                     "peak_source": "2 x measured bf16" if os.path.exists(peaks_path) else "fallback"}

    serving = None
    if world == 1 and args.serve_requests > 0:
        serving = run_serving(args, torch, polymul)
    uneven = None
    if world == 1 and args.uneven > 0:
        uneven = run_uneven(args, torch, polymul)
    special = run_special(args, torch, polymul, tuning) if world == 1 else None

    # K2 is bound by instruction issue, not by HBM: butterflies per second against the issue
    # bound of one warp instruction per SM sub-partition per clock (128 thread instructions
    # per SM per clock) at 7 instructions per lazy Harvey butterfly (2 IADD, 1 IMNMX,
    # 3 IMAD incl. the high product, 1 IADD3), at the clock sampled during the timed region
    alu = None
    if "k2_rows" in prof:
        cnt, tot = prof["k2_rows"]
        logr = 4 if args.path == "tensor" else 5
        rows_stages = (n.bit_length() - 1) - logr
        bfly = 3 * plan.primes * (n // 2) * rows_stages  # a, b forward + inverse, row stages only
        sms = torch.cuda.get_device_properties(local).multi_processor_count
        mhz = clocks.get("sm_mhz") or 1965.0
        peak_bfly = 128.0 / 7.0 * sms * mhz * 1e6
        achieved = bfly * timed_products / (tot / 1000.0)
        # the integer multiplier (fmaheavy pipe) bound: a butterfly's three multiplies hold it
        # 2 + 4 (the high product) + 2 cycles per warp, one pipe per SM sub-partition
        peak_mul = 32.0 / 8.0 * 4 * sms * mhz * 1e6
        alu = {"kernel": "k2_rows", "butterflies_per_product": bfly, "achieved_per_s": achieved,
               "peak_per_s": peak_bfly, "frac": achieved / peak_bfly,
               "unit": "butterflies/s", "sm_mhz": mhz,
               "model": "issue bound: 7 thread instructions per lazy butterfly, 128 per SM per clock",
               "multiplier_bound": {"peak_per_s": peak_mul, "frac": achieved / peak_mul,
                                    "model": "fmaheavy pipe: 8 cycles per warp-butterfly (IMAD 2 + IMAD.HI 4 + "
                                             "IMAD 2), 4 sub-partitions per SM"}}

    cpu = None
    if rank == 0 and world == 1 and args.cpu_seconds > 0:
        from tests import reference_emulation as emu

        cores = host_cores()
        (ca, cb), = host_inputs(n, q, args.seed + 5)
        threads = os.cpu_count() or 1
        v, done, el = cpu_sample(ca, cb, q, args.cpu_seconds, threads)
        port = {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                "sample": f"{done} products (N={n}, {bits}-bit q) in {el:.1f} s through the C restatement of the "
                          "reference RNS method (oracle/polymul_oracle.c), threads over primes"}
        if emu.available() and n <= 32768:
            # the reference's own kernels, one product per host core at once (the emulation is single-threaded)
            ev, wall, secs, (ea, eb, ec) = emulated_reference_sample(n, cores, cores, args.seed + 7)
            if not (ec == oracle.rns_multiply(ea, eb, FHERMA_Q)).all():
                raise SystemExit("emulated reference disagrees with the oracle")
            cpu = {"value": ev, "unit": UNIT, "cores": cores, "kind": "reference",
                   "sample": f"{cores} products (N={n}, q = 2^868 - 11993087, the form the reference takes) in "
                             f"{wall:.1f} s through the reference's own rns kernels run by its CPU emulation, one "
                             "single-threaded process per core", "port": port}
        else:
            cpu = port

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": {"workload": f"batch of {B} independent negacyclic products per step, N={n}, {bits}-bit "
                                   f"seeded odd q, coefficients uniform in [0, q) generated on the device",
                       "n": n, "q_bits": bits, "batch": B, "primes": plan.primes,
                       "path": args.path,
                       "l2": f"inputs larger than L2: {2 * B * io / 1e9:.2f} GB of a, b read per step",
                       "parallelism": f"replicas x{world}", "oracle_check": f"{checked} products bit-exact",
                       "tuning": tuning},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 2 * E * io, "d2h_bytes_per_step": E * io,
                    "api": "pm_multiply_host_batch, pinned host buffers", "products_per_step": E,
                    "link": link},
            "gpu_launches": launches,
            "roofline": roofline,
            "alu_roofline": alu,
            "tensor_pipe": tensor_pipe,
            "kernels": kernels,
            "cpu_baseline": cpu,
            "serving": serving,
            "batched_uneven": uneven,
            "plain": plain,
            "special_form_q": special,
            "clocks": clocks,
            "mismatches": mismatches,
        }
        print(json.dumps(line), flush=True)
    plan.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_ncu_case(args):
    """K single products of the benchmark workload, for `ncu -k ... -s ... -c ...` captures."""
    import torch

    import polymul

    torch.cuda.set_device(0)
    q = seeded_q(args.seed, args.bits)
    limbs = (args.bits + 63) // 64
    a = device_inputs(torch, args.ncu_case, args.ring, limbs, q, args.seed + 17)
    b = device_inputs(torch, args.ncu_case, args.ring, limbs, q, args.seed + 29)
    c = torch.empty_like(a)
    plan = polymul.Plan(args.ring, q, coef_limbs=limbs, tensor=(args.path == "tensor"))
    # one batched call, all K products in one launch group (one launch per pass)
    plan.set_tuning(group=args.ncu_case, conv_whole_basis=int(args.conversion == "whole"))
    plan.multiply_batch(a.data_ptr(), b.data_ptr(), c.data_ptr(), args.ncu_case)
    torch.cuda.synchronize()
    plan.close()
    print(f"ncu case: {args.ncu_case} products in one batched call, N={args.ring}, {args.bits}-bit q, "
          f"path {args.path}, conversion {args.conversion}")


def main():
    args = parse()
    if args.ncu_case:
        run_ncu_case(args)
        return
    if args.impl == "reference":
        run_reference(args)
        world, _, _ = dist_env()
        return
    run_ours(args)


if __name__ == "__main__":
    main()
