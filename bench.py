"""Decode benchmark of the B200 FastLanes engine.

Workload (one step): the batched bit-width sweep -- 65,536 u32 vectors (64 Mi values) + 32,768 u64 vectors
(32 Mi values), per-vector bit width uniform in 0..W and base uniform in [0, 2^W - 2^bw], values
base + U[0, 2^bw), both widths interleaved in one shuffled work queue and decoded (unpack + FOR add) in ONE
persistent kernel launch.  Inputs (~0.4 GB packed) and outputs (768 MiB) are far larger than the 126 MB L2,
so no flush is needed between timed steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  Under torchrun each rank decodes its own copy (weak scaling, no collective on
the data path); time is the max over ranks of the device-timed region.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "decoded GB/s, % HBM roofline"
WORKLOAD = "batched bit-width sweep: 64Mi u32 + 32Mi u64 FFOR vectors, bw~U{0..W}, shuffled, 1 persistent launch"
N32, N64 = 65536, 32768


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="budget of the CPU baseline sample")
    return ap.parse_args()


def dist_setup(args):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    return world, rank, local


class ClockSampler:
    """nvidia-smi clocks + throttle reasons sampled every 200 ms while the timed region runs."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows if len(r) > 8 for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def gpu_id(dev):
    """nvidia-smi id of a torch device (its UUID, which survives CUDA_VISIBLE_DEVICES remapping)."""
    import torch

    try:
        u = str(torch.cuda.get_device_properties(dev).uuid)
        return u if u.startswith("GPU-") else "GPU-" + u
    except Exception:
        return str(dev.index or 0)


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic():
    """Per-launch DRAM bytes of the decode kernel from the committed ncu summary, if one exists."""
    try:
        with open(os.path.join(ROOT, "profiles", "decode_bw_sweep_traffic.json")) as f:
            return json.load(f)
    except Exception:
        return None


def host_columns(columns, n32, n64):
    """First n32 u32 / n64 u64 vectors of device columns, copied to the host for the CPU leg."""
    out = []
    for c, n in zip(columns, (n32, n64)):
        off = c.byte_off[:n].cpu().numpy()
        end = int(off[-1]) + int(c.bw[n - 1].item()) * 128
        out.append((c.width, c.packed[: end + 64].cpu().numpy(), off, c.bw[:n].cpu().numpy(),
                    c.base[:n].cpu().numpy().view(np.uint8)))
    return out


def cpu_reference_leg(host, seconds, kind):
    """The reference's own unffor (oracle/_ref, compiled from its sources) -- or the oracle port where the
    reference library is absent -- over a bounded sample of the workload's vectors, on all host cores."""
    import ctypes

    from oracle import oracle as orc

    lib = orc.reference if (kind == "reference" and orc.reference is not None) else None
    port = lib is None
    cores = os.cpu_count() or 1
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    # sample: the first S vectors of each width in the same 2:1 proportion as the workload
    S = 2048 if not port else 64
    host = [(w, pk, off[:S if w == 32 else S // 2], bw[:S if w == 32 else S // 2], base) for (w, pk, off, bw, base)
            in host]
    done_vals, done_bytes, t_total = 0, 0, 0.0
    reps = 0
    while t_total < seconds and reps < 1000:
        for (w, pk, off, bw, base) in host:
            n = min(S if w == 32 else S // 2, bw.size)
            out = np.empty(n * 1024 * w // 8, np.uint8)
            t0 = time.perf_counter()
            if port:
                lo = orc.lib()
                lo.fls_o_unffor_batch_bytes(ctypes.c_int(w), P(pk), P(off), P(bw), P(base), ctypes.c_uint64(0),
                                            ctypes.c_uint64(n), P(out))
            else:
                lib.ref_unffor_batch(ctypes.c_int(w), P(pk), P(off), P(bw), P(base), ctypes.c_uint64(n), P(out),
                                     ctypes.c_int(cores))
            t_total += time.perf_counter() - t0
            done_vals += n * 1024
            done_bytes += n * 1024 * w // 8
        reps += 1
    return {"value": round(done_bytes / t_total / 1e9, 3), "unit": "GB/s",
            "values_per_s": done_vals / t_total, "cores": 1 if port else cores,
            "kind": "port" if port else "reference",
            "sample": f"{reps} passes over the first {S} u32 + {S // 2} u64 vectors of the workload "
                      f"({t_total:.1f} s of decode)"}


def cpu_sample(seed, n32, n64):
    """Host-side sample of the workload for the reference arm, encoded with the reference's own ffor
    (generated::ffor::fallback::scalar::ffor) after its own transpose_i -- no GPU and no code of this
    engine on that path."""
    import ctypes

    from oracle import oracle as orc

    ref = orc.reference
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    rng = np.random.default_rng(seed)
    out = []
    for w, n in ((32, n32), (64, n64)):
        T = np.uint32 if w == 32 else np.uint64
        bw = rng.integers(0, w + 1, n).astype(np.uint8)
        chunks, offs, bases, pos = [], [], [], 0
        for v in range(n):
            b = int(bw[v])
            hi = (1 << w) - (1 << b)
            base = T(int(rng.integers(0, hi, dtype=np.uint64, endpoint=True)) if hi > 0 else 0)
            x = rng.integers(0, np.iinfo(np.uint64).max, 1024, dtype=np.uint64, endpoint=True)
            if b < 64:
                x &= np.uint64((1 << b) - 1)
            x = (x.astype(T) + base).astype(T)
            tr = np.empty_like(x)
            getattr(ref, f"ref_transpose_i_u{w}")(P(x), P(tr))
            pk = np.zeros(1024, T)
            getattr(ref, f"ref_ffor_u{w}")(P(tr), P(pk), ctypes.c_uint8(b), P(np.array([base], T)))
            chunks.append(pk[: b * 1024 // w].view(np.uint8))
            offs.append(pos)
            pos += b * 128
            bases.append(base)
        out.append((w, np.concatenate(chunks + [np.zeros(64, np.uint8)]), np.array(offs, np.uint64), bw,
                    np.array(bases, T).view(np.uint8)))
    return out


def run_reference(args):
    """Reference arm: the reference's own CPU unffor on the box's host cores (rank 0 only, no GPU)."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    from oracle import oracle as orc

    if orc.reference is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libfls_ref.so (the reference compiled "
                                                              "from its sources) is not present"}), flush=True)
        return
    host = cpu_sample(0, 2048, 1024)
    per_step = []
    for i in range(args.warmup + args.steps):
        leg = cpu_reference_leg(host, max(args.cpu_seconds / max(args.steps, 1), 0.2), "reference")
        if i >= args.warmup:
            per_step.append(leg)
    val = float(np.median([s["value"] for s in per_step]))
    line = {"impl": "reference", "metric": METRIC, "value": round(val, 3), "unit": "GB/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32+u64", "data": "synthetic (seeded)",
            "config": {"workload": WORKLOAD, "host_cores": per_step[-1]["cores"]},
            "cpu_baseline": {k: per_step[-1][k] for k in ("kind", "cores", "sample")} | {"value": round(val, 3),
                                                                                         "unit": "GB/s"},
            "e2e": {"value": round(val, 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args):
    import torch

    world, rank, local = dist_setup(args)
    from fastlanes_b200 import _lib, workloads
    from fastlanes_b200 import primitives as P

    dev = torch.device("cuda", local if world > 1 else 0)
    cols, queue = workloads.bw_sweep(N32, N64, seed=rank, device=dev, keep_values=True)
    outs = [torch.empty(c.n_vec * 1024, dtype=workloads._DT[c.width], device=dev) for c in cols]
    plan_t = workloads.Plan(cols, outs, order=P.TRANSPOSED, queue=queue)
    plan_o = workloads.Plan(cols, outs, order=P.ORIGINAL, queue=queue)
    plan_k = workloads.Plan(cols, outs, order=P.TRANSPOSED, queue=queue, keep_order=True)

    # correctness guard: original-order decode must reproduce the generated values exactly
    plan_o.decode()
    torch.cuda.synchronize()
    for c, o in zip(cols, outs):
        if not torch.equal(o.view(torch.int64 if c.width == 64 else torch.int32),
                           c.values.view(torch.int64 if c.width == 64 else torch.int32)):
            raise SystemExit("decode mismatch in benchmark self-check")
        c.values = None
    if P.device_status() != 0:
        raise SystemExit("device status error")

    read_b = sum(c.algorithmic_read_bytes() for c in cols) + queue.numel() * 4
    write_b = sum(c.decoded_bytes() for c in cols)
    n_vals = sum(c.n_vec * 1024 for c in cols)
    stream = torch.cuda.current_stream()

    def timed(plan, steps, warm):
        for _ in range(warm):
            plan.decode()
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        _lib.lib.fls_gpu_launch_count(1)
        ev0.record(stream)
        for _ in range(steps):
            plan.decode()
        ev1.record(stream)
        torch.cuda.synchronize()
        launches = _lib.lib.fls_gpu_launch_count(1)
        ms = ev0.elapsed_time(ev1) / steps
        if world > 1:
            t = torch.tensor([ms], device=dev)
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            ms = float(t.item())
            torch.distributed.barrier()
        return ms, launches

    with ClockSampler(gpu_id(dev)) as clk:
        ms_t, launches = timed(plan_t, args.steps, args.warmup)
        ms_o, _ = timed(plan_o, max(args.steps // 2, 3), 3)
        ms_k, _ = timed(plan_k, max(args.steps // 4, 3), 3)
    clocks = clk.summary()

    # end to end through the public API: host (pinned) -> device copy of the compressed inputs, one decode,
    # device -> host copy of the decoded values, every step
    h_in = [(c.packed.cpu().pin_memory(), c.byte_off.cpu().pin_memory(), c.bw.cpu().pin_memory(),
             c.base.cpu().pin_memory()) for c in cols]
    h_out = [torch.empty(o.numel(), dtype=o.dtype, pin_memory=True) for o in outs]
    h2d = sum(sum(t.numel() * t.element_size() for t in hi) for hi in h_in) + queue.numel() * 4
    h_q = queue.cpu().pin_memory()
    d2h = sum(o.numel() * o.element_size() for o in outs)

    def e2e_step():
        for (hp, ho, hb, hs), c in zip(h_in, cols):
            c.packed.copy_(hp, non_blocking=True)
            c.byte_off.copy_(ho, non_blocking=True)
            c.bw.copy_(hb, non_blocking=True)
            c.base.copy_(hs, non_blocking=True)
        queue.copy_(h_q, non_blocking=True)
        plan_o.decode()
        for o, ho in zip(outs, h_out):
            ho.copy_(o, non_blocking=True)

    for _ in range(2):
        e2e_step()
    torch.cuda.synchronize()
    e_steps = max(3, min(args.steps, 10))
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(e_steps):
        e2e_step()
    ev1.record(stream)
    torch.cuda.synchronize()
    e_ms = ev0.elapsed_time(ev1) / e_steps
    if world > 1:
        t = torch.tensor([e_ms], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e_ms = float(t.item())

    cpu = None
    if rank == 0 and world == 1:
        cpu = cpu_reference_leg(host_columns(cols, 2048, 1024), args.cpu_seconds, "reference")

    if rank == 0:
        peak, peak_src = measured_peak()
        achieved = (read_b + write_b) / (ms_t * 1e-3) / 1e9
        value = write_b * world / (ms_t * 1e-3) / 1e9
        traffic = profiled_traffic()
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_t, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32+u64", "data": "synthetic (seeded; values base+U[0,2^bw))",
            "config": {"workload": WORKLOAD, "vectors": N32 + N64, "values": n_vals, "order": "transposed",
                       "queue": "shuffled; planner groups items by vector width (data untouched)",
                       "l2": "inputs and outputs larger than L2, no flush", "parallelism": f"replicas{world}"},
            "decoded_values_per_s": round(n_vals * world / (ms_t * 1e-3), 1),
            "queue_as_shuffled": {"ms_per_step": round(ms_k, 4),
                                  "value": round(write_b * world / (ms_k * 1e-3) / 1e9, 2), "unit": "GB/s",
                                  "note": "planner grouping of work items by vector width switched off"},
            "original_order": {"ms_per_step": round(ms_o, 4),
                               "value": round(write_b * world / (ms_o * 1e-3) / 1e9, 2), "unit": "GB/s"},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "peak_source": peak_src,
                         "bytes_per_launch": read_b + write_b,
                         "traffic": (traffic or {}).get("bytes_per_launch")},
            "cpu_baseline": cpu,
            "e2e": {"value": round(write_b * world / (e_ms * 1e-3) / 1e9, 3), "unit": "GB/s",
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "ms_per_step": round(e_ms, 3)},
            "clocks": clocks,
            "gpu_launches": int(launches),
        }
        print(json.dumps(line), flush=True)
    plan_t.close()
    plan_o.close()
    plan_k.close()
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
