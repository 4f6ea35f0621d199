#!/usr/bin/env python
"""Benchmark of the B200 ZB2 block codec: compress then extract (a bit-exact round trip) of 1 GiB of
LZ-structured synthetic data per GPU at block 2^18 (256 KiB) and level 5.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
    python -m torch.distributed.run --nproc-per-node N --master-addr 127.0.0.1 bench.py --gpus N ...

One step = compress the whole input (one launch per stage per 256 MiB of blocks) and decompress the
result, all device-resident: `value` is raw GB / step time over every rank (max over ranks of the device
time).  `e2e` is the same round trip through the host C ABI (zc_compress / zc_decompress) with pinned host
buffers, copies included.  Per-kernel CUDA-event times give the dominant kernel's roofline against the
measured HBM bandwidth; the reference CPU codec (oracle/_ref, all host threads) is timed on a sample.

Blocks are independent, so N GPUs each code their own 1 GiB (weak scaling, no collective on the data
path; a barrier and a max-reduction of the timings only).

--impl reference times the reference's own CPU codec (CpuCodec of src/archive.h, compiled from the
reference sources into oracle/_ref/libzref.so; the C restatement oracle/liboracle.so when that is absent)
on a bounded sample of the same workload, on rank 0 only.
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
sys.path.insert(0, os.path.join(ROOT, "zero-compression_b200"))

METRIC = "compress/decompress GB/s on 1 B200, bit-exact round-trip; served p50/p99 latency"
# dram__bytes_read.sum + dram__bytes_write.sum per raw byte of one launch (block 18, level 5 lz_mix), from
# the ncu captures summarised in profiles/encoder_kernels_lz256m_b18_l5.md (256 MiB launch),
# profiles/decoder_fill_lz512m_b18_l5.md (512 MiB launch) and profiles/decoder_kernels_lz256m_b18_l5.md
DRAM_BYTES_PER_RAW_BYTE = {"k_enc_match": 10.893, "k_enc_parse": 24.74, "k_sort_scatter": 9.81,
                           "k_dec_fill": 2.084, "k_dec_tokens": 0.186, "k_dec_streams": 0.198}
GB = 1e9


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while the timed region runs."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
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
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.t.join(timeout=2)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            if len(r) > 8:
                for k, nm in enumerate(names):
                    if r[5 + k].lower().startswith("active"):
                        reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def make_data(n, block_log, seed):
    import datagen as G
    return G.lz_mix(n, block_log, seed)


def cpu_round_trip(data, block_log, level):
    """One round trip of `data` through the reference CPU codec (all threads); returns (seconds, kind, cores)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import oracle as O
    B = 1 << block_log
    if O.Ref.available():
        t0 = time.perf_counter()
        methods, lens, pays = O.Ref.cpu_compress(data, block_log, O.depth_for_level(level))
        comp, offs, at = [], [], 0
        for b in range(len(methods)):
            blk = data[b * B:(b + 1) * B]
            c = pays[b] if methods[b] else blk.tobytes()
            comp.append(c)
            offs.append(at)
            at += len(c)
        raw_lens = [min(B, data.size - b * B) for b in range(len(methods))]
        blob = np.frombuffer(b"".join(comp), np.uint8)
        out = O.Ref.cpu_decompress(blob, offs, [len(c) for c in comp], methods, raw_lens)
        dt = time.perf_counter() - t0
        assert np.array_equal(out, data), "reference CPU round trip differs"
        return dt, "reference", O.Ref.hardware_threads()
    if not O.Port.available():
        O.build()
    t0 = time.perf_counter()
    for o in range(0, data.size, B):
        blk = data[o:o + B].tobytes()
        pay = O.Port.compress_block(blk, O.depth_for_level(level))
        if len(pay) < len(blk):
            assert O.Port.decompress_block(pay, len(blk)) == blk
    return time.perf_counter() - t0, "port", 1


def run_reference(args):
    ws, rank, local = dist_env()
    if rank != 0:
        return 0
    B = 1 << args.block
    sample = min(args.size_mib << 20, 256 << 20)
    data = make_data(sample, args.block, 1000)
    times = []
    kind, cores = "reference", 1
    for i in range(args.warmup + args.steps):
        dt, kind, cores = cpu_round_trip(data, args.block, args.level)
        if i >= args.warmup:
            times.append(dt)
    t = statistics.mean(times)
    value = sample / t / GB
    desc = f"{sample >> 20} MiB of the lz_mix workload (block {B >> 10} KiB, level {args.level}), round trip per step"
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": "GB/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(t * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded lz_mix generator)",
        "config": dict(workload_config(args), sample_bytes=sample,
                       workload=f"lz_mix {args.size_mib} MiB per GPU (each step times a {sample >> 20} MiB sample of "
                                f"it on the host cores), block {args.block} ({B >> 10} KiB), level {args.level}: "
                                f"compress then extract (bit-exact round trip)"),
        "cpu_baseline": {"value": round(value, 4), "unit": "GB/s", "cores": cores, "kind": kind, "sample": desc},
        "e2e": {"value": round(value, 4), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def workload_config(args):
    return {"workload": f"lz_mix {args.size_mib} MiB per GPU, block {args.block} ({(1 << args.block) >> 10} KiB), "
                        f"level {args.level}: compress then extract (bit-exact round trip)",
            "block_log": args.block, "level": args.level, "bytes_per_gpu": args.size_mib << 20,
            "generator": "literal runs geometric(mean 8) over geometric(p=0.05) symbols; matches log-uniform "
                         "length [4,258], offset log-uniform [1, block]",
            "l2_flush": "none needed: 1 GiB of input per GPU is larger than the 126 MB L2",
            "parallelism": f"dp{args.gpus} (independent blocks per GPU)"}


def run_ours(args):
    import numpy as np
    import torch
    import torch.distributed as dist
    import zero_cuda as Z

    ws, rank, local = dist_env()
    if ws > 1:
        torch.cuda.set_device(local)
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)

    bl, level = args.block, args.level
    B = 1 << bl
    n = args.size_mib << 20
    nb = (n + B - 1) // B
    host = make_data(n, bl, 1000 + rank)
    pinned = torch.empty(n, dtype=torch.uint8, pin_memory=True)
    pinned.numpy()[:] = host
    codec = Z.CudaCodec(level=level, device=local)
    per = codec.batch_bytes(bl) // B  # blocks per launch

    d_in = torch.zeros(n + 64, dtype=torch.uint8, device=dev)
    d_in[:n].copy_(pinned, non_blocking=False)
    offs = torch.arange(nb, dtype=torch.int64, device=dev) * B
    lens = torch.clamp(n - offs, max=B).to(torch.int32)
    d_out = torch.empty(n + 64, dtype=torch.uint8, device=dev)
    d_dec = torch.empty(n + 64, dtype=torch.uint8, device=dev)
    methods = torch.zeros(nb, dtype=torch.uint8, device=dev)
    clens = torch.zeros(nb, dtype=torch.int32, device=dev)
    crcs = torch.zeros(nb, dtype=torch.int32, device=dev)
    dcrcs = torch.zeros(nb, dtype=torch.int32, device=dev)
    errs = torch.zeros(nb, dtype=torch.int32, device=dev)
    ooffs = torch.zeros(nb, dtype=torch.int64, device=dev)
    totals = torch.zeros((nb + per - 1) // per, dtype=torch.int64, device=dev)
    stream = torch.cuda.Stream(device=dev)
    sh = stream.cuda_stream
    chunks = [(b0, min(per, nb - b0)) for b0 in range(0, nb, per)]

    chunk_base = torch.tensor([b0 * B for b0, k in chunks for _ in range(k)], dtype=torch.int64, device=dev)
    goffs = torch.zeros(nb, dtype=torch.int64, device=dev)
    dec_per = codec.batch_bytes_decode(bl) // B  # blocks per decoder launch

    def compress():
        # one launch per stage per chunk of blocks; each chunk's record bodies land in its own slice of d_out
        for ci, (b0, k) in enumerate(chunks):
            o = b0 * B
            codec.compress_device(d_in, offs[b0:], lens[b0:], k, bl, methods[b0:], clens[b0:], crcs[b0:],
                                  d_out[o:o + k * B + 64], ooffs[b0:], totals[ci:], stream=sh)
        with torch.cuda.stream(stream):
            torch.add(ooffs, chunk_base, out=goffs)  # record offsets from the start of d_out

    def decompress():
        for b0 in range(0, nb, dec_per):
            k = min(dec_per, nb - b0)
            codec.decompress_device(d_out, goffs[b0:], clens[b0:], methods[b0:], lens[b0:], k, bl, d_dec, offs[b0:],
                                    dcrcs[b0:], errs[b0:], stream=sh)

    def barrier():
        if ws > 1:
            dist.barrier()

    # warm-up (untimed)
    for _ in range(args.warmup):
        compress()
        decompress()
    torch.cuda.synchronize(dev)
    comp_bytes = int(totals.sum().item())

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
           torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    codec.profile(True)
    launches0 = codec.launch_count()
    barrier()
    torch.cuda.synchronize(dev)
    with ClockSampler(local) as clk:
        with torch.cuda.stream(stream):
            for i in range(args.steps):
                ev[i][0].record(stream)
                compress()
                ev[i][1].record(stream)
                decompress()
                ev[i][2].record(stream)
        torch.cuda.synchronize(dev)
    barrier()
    launches = codec.launch_count() - launches0
    stages = codec.profile_stages()
    codec.profile(False)
    t_c = [ev[i][0].elapsed_time(ev[i][1]) for i in range(args.steps)]
    t_d = [ev[i][1].elapsed_time(ev[i][2]) for i in range(args.steps)]
    tot_ms = ev[0][0].elapsed_time(ev[-1][2])
    local_times = torch.tensor([tot_ms, sum(t_c), sum(t_d)], dtype=torch.float64, device=dev)
    if ws > 1:
        dist.all_reduce(local_times, op=dist.ReduceOp.MAX)
    tot_ms, sum_c, sum_d = local_times.tolist()

    # bit-exact round trip and CRCs
    ok = bool(torch.equal(d_dec[:n], d_in[:n])) and bool(torch.equal(dcrcs, crcs)) and int(errs.abs().sum()) == 0
    flags = torch.tensor([0 if ok else 1], device=dev)
    if ws > 1:
        dist.all_reduce(flags, op=dist.ReduceOp.MAX)
    ok = int(flags.item()) == 0

    ms_per_step = tot_ms / args.steps
    value = ws * n / (ms_per_step * 1e-3) / GB
    comp_gbs = ws * n / (sum_c / args.steps * 1e-3) / GB
    dec_gbs = ws * n / (sum_d / args.steps * 1e-3) / GB

    # the dominant kernel: most time in the timed region; its algorithmic bytes are the codec's
    # (raw + compressed) bytes of the blocks one launch covers
    peak, peak_kind = peaks()
    dom = max(stages.items(), key=lambda kv: kv[1][0]) if stages else ("", (0.0, 1))
    dom_name, (dom_ms, dom_launches) = dom
    steps_bytes = (n + comp_bytes) * args.steps
    achieved = steps_bytes / (dom_ms * 1e-3) / GB if dom_ms else 0.0
    # DRAM traffic of one launch: ncu's dram bytes per raw byte for the kernel (a capture of the same
    # kernel on a smaller launch; traffic grows with the blocks processed), times the raw bytes per launch
    per_byte = DRAM_BYTES_PER_RAW_BYTE.get(dom_name)
    traffic = int(per_byte * n / max(1, dom_launches // args.steps)) if per_byte else None
    total_stage_ms = sum(v[0] for v in stages.values()) or 1.0
    pipe_achieved = steps_bytes / (tot_ms * 1e-3) / GB

    line = {
        "metric": METRIC, "value": round(value, 4), "unit": "GB/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded lz_mix generator, 1 GiB per GPU)",
        "config": workload_config(args),
        "compress_gbs": round(comp_gbs, 4), "decompress_gbs": round(dec_gbs, 4),
        "ratio": round(comp_bytes / n, 5), "bit_exact": ok,
        "roofline": {"bound": "hbm", "kernel": dom_name, "achieved": round(achieved, 2), "peak": peak,
                     "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": traffic,
                     "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind,
                     "algorithmic_bytes_per_launch": int((n + comp_bytes) / max(1, dom_launches // args.steps)),
                     "avg_launch_ms": round(dom_ms / max(1, dom_launches), 4),
                     "pipeline_frac": round(pipe_achieved / peak, 4)},
        "stages_ms_per_step": {k: round(v[0] / args.steps, 4) for k, v in stages.items()},
        "stage_share": {k: round(v[0] / total_stage_ms, 4) for k, v in stages.items()},
        "gpu_launches": int(launches),
    }

    # end to end through the host C ABI with pinned buffers (rank-local wall time, max over ranks)
    pay_p = torch.empty(n + 64, dtype=torch.uint8, pin_memory=True)
    dec_p = torch.empty(n + 64, dtype=torch.uint8, pin_memory=True)
    m_h = np.zeros(nb, np.uint8)
    l_h = np.zeros(nb, np.uint32)
    c_h = np.zeros(nb, np.uint32)
    o_h = np.zeros(nb, np.uint64)
    raw_lens = np.minimum(B, n - np.arange(nb, dtype=np.int64) * B).astype(np.uint32)
    hin = pinned.numpy()

    def e2e_step():
        codec.compress_arrays(hin, bl, out=(m_h, l_h, c_h, pay_p.numpy(), o_h))
        # the record bodies as an archive holds them: each payload, or the raw block when stored
        # (stored blocks are appended after the payloads, as a reader would hand them over)
        pay_total = int(l_h[m_h == 1].sum())
        comp_offs = o_h.copy()
        at = pay_total
        pv = pay_p.numpy()
        for b in np.nonzero(m_h == 0)[0]:
            pv[at:at + raw_lens[b]] = hin[b * B: b * B + raw_lens[b]]
            comp_offs[b] = at
            at += int(raw_lens[b])
        codec.decompress_arrays(pv, comp_offs, l_h, m_h, raw_lens, out=dec_p.numpy())
        return pay_total, at

    e2e = None
    try:
        for _ in range(1):
            e2e_step()
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            pay_total, body_total = e2e_step()
        dt = (time.perf_counter() - t0) / args.steps
        dts = torch.tensor([dt], dtype=torch.float64, device=dev)
        if ws > 1:
            dist.all_reduce(dts, op=dist.ReduceOp.MAX)
        dt = float(dts.item())
        same = bool(np.array_equal(dec_p.numpy()[:n], hin))
        # compress: n bytes up, per-block records (17 B) and payloads down; decompress: the record bodies
        # and a 33-byte block table up, n bytes and per-block CRC + status (8 B) down
        e2e = {"value": round(ws * n / dt / GB, 4), "unit": "GB/s",
               "h2d_bytes_per_step": int(n + body_total + nb * 33), "d2h_bytes_per_step": int(pay_total + n + nb * 25),
               "bit_exact": same, "path": "zc_compress + zc_decompress, pinned host buffers"}
    except Exception as e:  # reported, never hidden
        e2e = {"value": None, "unit": "GB/s", "error": str(e)[:200]}
    line["e2e"] = e2e
    line["clocks"] = clk.summary()

    if rank == 0 and ws == 1 and not args.no_cpu:
        sample = host[: min(n, 256 << 20)]
        reps, t_cpu, kind, cores = 0, 0.0, "reference", 1
        while reps < 1 or (t_cpu < 5.0 and reps < 8):
            dt, kind, cores = cpu_round_trip(sample, bl, level)
            t_cpu += dt
            reps += 1
        line["cpu_baseline"] = {"value": round(sample.size * reps / t_cpu / GB, 4), "unit": "GB/s", "cores": cores,
                                "kind": kind,
                                "sample": f"{sample.size >> 20} MiB of the same input, compress + decompress, "
                                          f"{reps} round trip(s), block {B >> 10} KiB, level {level}"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    codec.close()
    if ws > 1:
        dist.destroy_process_group()
    return 0 if ok else 1


def _events(n):
    import torch
    return [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(n)]


def run_batched(args):
    """Many-file workload (the batched-archive config, scaled): files of log-uniform sizes, each cut into
    blocks with its own short tail, generators drawn from the text mix, the LZ mix and random bytes.
    Plain form: one compress and one decompress call per file.  Batched form: blocks of many files in one
    call per stage (up to the launch capacity), replayed as CUDA graphs.  Device-resident, bit-exact."""
    import numpy as np
    import torch
    import zero_cuda as Z
    import datagen as G
    ws, rank, local = dist_env()
    if rank != 0:
        return 0
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    bl, level = args.block, args.level
    B = 1 << bl
    sizes, kinds = G.file_plan(args.files, 1 << 10, args.max_file_kib << 10, seed=2024)
    sizes = sizes.astype(np.int64)
    file_off = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
    total = int(sizes.sum())
    pinned = torch.empty(total + 64, dtype=torch.uint8, pin_memory=True)
    hv = pinned.numpy()
    from concurrent.futures import ThreadPoolExecutor

    def gen(f):  # (the generators run in C without the interpreter lock: host threads fill files side by side)
        o, n = int(file_off[f]), int(sizes[f])
        k = int(kinds[f])
        out = hv[o:o + n]
        if k == 0:
            G.text_mix(n, 5000 + f, out=out)
        elif k == 1:
            G.lz_mix(n, bl, 5000 + f, out=out)
        else:
            G.random_bytes(n, 5000 + f, out=out)

    with ThreadPoolExecutor(16) as ex:
        list(ex.map(gen, range(args.files)))
    # block list: each file's blocks, its last one short
    nblk = (sizes + B - 1) // B
    first = np.concatenate([[0], np.cumsum(nblk)[:-1]]).astype(np.int64)
    nb = int(nblk.sum())
    boffs = np.concatenate([file_off[f] + np.arange(nblk[f], dtype=np.int64) * B for f in range(args.files)])
    blens = np.concatenate([np.minimum(B, sizes[f] - np.arange(nblk[f], dtype=np.int64) * B)
                            for f in range(args.files)]).astype(np.int32)
    d_in = torch.zeros(total + 64, dtype=torch.uint8, device=dev)
    d_in.copy_(pinned)
    del pinned, hv
    offs = torch.tensor(boffs, device=dev)
    lens = torch.tensor(blens, device=dev)
    d_out = torch.zeros(total + 64, dtype=torch.uint8, device=dev)
    codec = Z.CudaCodec(level=level, device=local)
    per = codec.batch_bytes(bl) // B
    dper = codec.batch_bytes_decode(bl) // B
    if args.chunk_mib:  # smaller launches: less scratch (the full-size set must fit beside its input and output)
        per = max(1, min(per, (args.chunk_mib << 20) // B))
        dper = max(1, min(dper, (2 * args.chunk_mib << 20) // B))
    # Decoded bytes: in place of the input's layout when it fits beside everything else; else into one
    # buffer of a decode batch (or the largest file), each batch's and file's blocks from its start, checked
    # against the input after the timed steps.
    small = total <= (24 << 30)
    dec_cap = total if small else max(dper * B, int(sizes.max()))
    d_dec = torch.zeros(dec_cap + 64, dtype=torch.uint8, device=dev)
    if small:
        offs_dec, offs_file = offs, offs
    else:
        bidx = np.arange(nb, dtype=np.int64)
        offs_dec = torch.tensor(boffs - boffs[(bidx // dper) * dper], device=dev)
        offs_file = torch.tensor(boffs - np.repeat(file_off, nblk), device=dev)
    methods = torch.zeros(nb, dtype=torch.uint8, device=dev)
    clens = torch.zeros(nb, dtype=torch.int32, device=dev)
    crcs = torch.zeros(nb, dtype=torch.int32, device=dev)
    dcrcs = torch.zeros(nb, dtype=torch.int32, device=dev)
    errs = torch.zeros(nb, dtype=torch.int32, device=dev)
    ooffs = torch.zeros(nb, dtype=torch.int64, device=dev)
    goffs = torch.zeros(nb, dtype=torch.int64, device=dev)
    totals = torch.zeros(max(args.files, nb) + 1, dtype=torch.int64, device=dev)
    stream = torch.cuda.Stream(device=dev)
    sh = stream.cuda_stream
    chunks = [(b0, min(per, nb - b0)) for b0 in range(0, nb, per)]
    chunk_base = torch.tensor(np.concatenate([np.full(k, boffs[b0], np.int64) for b0, k in chunks]), device=dev)

    # per-file arguments as raw device addresses, computed once (keeps Python out of the measured loop)
    P = {name: t.data_ptr() for name, t in dict(d_in=d_in, offs=offs, lens=lens, methods=methods, clens=clens,
                                                 crcs=crcs, d_out=d_out, ooffs=ooffs, totals=totals, d_dec=d_dec,
                                                 dcrcs=dcrcs, errs=errs, offs_file=offs_file).items()}
    pc, pd = [], []
    for f in range(args.files):
        b0, k, o = int(first[f]), int(nblk[f]), int(file_off[f])
        pc.append((P["d_in"], P["offs"] + 8 * b0, P["lens"] + 4 * b0, k, bl, P["methods"] + b0, P["clens"] + 4 * b0,
                   P["crcs"] + 4 * b0, P["d_out"] + o, P["ooffs"] + 8 * b0, P["totals"] + 8 * f, int(sizes[f]) + 64))
        pd.append((P["d_out"] + o, P["ooffs"] + 8 * b0, P["clens"] + 4 * b0, P["methods"] + b0, P["lens"] + 4 * b0, k,
                   bl, P["d_dec"], P["offs_file"] + 8 * b0, P["dcrcs"] + 4 * b0, P["errs"] + 4 * b0))

    def plain_c():
        for a in pc:
            codec.compress_device(*a[:11], stream=sh, out_cap=a[11])

    def plain_d():
        for a in pd:
            codec.decompress_device(*a, stream=sh)

    def batched_c():
        for ci, (b0, k) in enumerate(chunks):
            o = int(boffs[b0])
            end = int(boffs[b0 + k - 1]) + int(blens[b0 + k - 1])
            codec.compress_device(d_in, offs[b0:], lens[b0:], k, bl, methods[b0:], clens[b0:], crcs[b0:],
                                  d_out[o:end + 64], ooffs[b0:], totals[ci:], stream=sh)
        with torch.cuda.stream(stream):
            torch.add(ooffs, chunk_base, out=goffs)

    def batched_d():
        for b0 in range(0, nb, dper):
            k = min(dper, nb - b0)
            codec.decompress_device(d_out, goffs[b0:], clens[b0:], methods[b0:], lens[b0:], k, bl, d_dec, offs_dec[b0:],
                                    dcrcs[b0:], errs[b0:], stream=sh)

    def bytes_equal(batched):
        """The decoded bytes against the input (every byte; batch by batch when decoded in place)."""
        if small:
            return bool(torch.equal(d_dec[:total], d_in[:total]))
        torch.cuda.synchronize(dev)
        if batched:
            for b0 in range(0, nb, dper):
                k = min(dper, nb - b0)
                o0, o1 = int(boffs[b0]), int(boffs[b0 + k - 1]) + int(blens[b0 + k - 1])
                batched_d_one(b0, k)
                torch.cuda.synchronize(dev)
                if not torch.equal(d_dec[:o1 - o0], d_in[o0:o1]):
                    return False
        else:
            for f in range(args.files):
                codec.decompress_device(*pd[f], stream=sh)
                torch.cuda.synchronize(dev)
                o = int(file_off[f])
                if not torch.equal(d_dec[:int(sizes[f])], d_in[o:o + int(sizes[f])]):
                    return False
        return True

    def batched_d_one(b0, k):
        codec.decompress_device(d_out, goffs[b0:], clens[b0:], methods[b0:], lens[b0:], k, bl, d_dec, offs_dec[b0:],
                                dcrcs[b0:], errs[b0:], stream=sh)

    def timed(fc, fd, label):
        for _ in range(args.warmup):
            fc(); fd()
        torch.cuda.synchronize(dev)
        ev = [_events(2) for _ in range(args.steps)]
        l0 = codec.launch_count()
        with torch.cuda.stream(stream):
            for i in range(args.steps):
                ev[i][0][0].record(stream); fc(); ev[i][0][1].record(stream)
                ev[i][1][0].record(stream); fd(); ev[i][1][1].record(stream)
        torch.cuda.synchronize(dev)
        tc = sum(e[0][0].elapsed_time(e[0][1]) for e in ev) / args.steps
        td = sum(e[1][0].elapsed_time(e[1][1]) for e in ev) / args.steps
        ok = bool(torch.equal(dcrcs, crcs)) and not errs.any() and bytes_equal(label == "batched")
        snap = (methods.clone(), clens.clone())
        d_dec.zero_()
        return {"compress_gbs": round(total / tc / 1e6, 3), "decompress_gbs": round(total / td / 1e6, 3),
                "round_trip_gbs": round(total / (tc + td) / 1e6, 3), "ms_compress": round(tc, 3),
                "ms_decompress": round(td, 3), "launches_per_step": (codec.launch_count() - l0) // args.steps,
                "bit_exact": ok}, snap

    # scratch at its largest first, so that graphs captured later stay valid
    batched_c(); batched_d(); torch.cuda.synchronize(dev)
    codec.set_graphs(False)
    plain, ps = timed(plain_c, plain_d, "plain")
    codec.set_graphs(True)
    batched, bs = timed(batched_c, batched_d, "batched")
    same = bool(torch.equal(ps[0], bs[0]) and torch.equal(ps[1], bs[1]))
    comp_bytes = int(clens.sum().item())
    line = {"metric": METRIC, "value": batched["round_trip_gbs"], "unit": "GB/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "dtype": "u8",
            "data": "synthetic (seeded per-file generators)",
            "config": {"workload": f"batched archive: {args.files} files, sizes log-uniform 1 KiB-{args.max_file_kib} "
                                   f"KiB ({total / 2**30:.2f} GiB), generators text/lz/random, block {bl}, level {level}",
                       "blocks": nb, "bytes": total, "encoder_launch_blocks": per, "decoder_launch_blocks": dper,
                       "decoded_in_place": small},
            "plain": plain, "batched": batched,
            "speedup_compress": round(batched["compress_gbs"] / plain["compress_gbs"], 3),
            "speedup_decompress": round(batched["decompress_gbs"] / plain["decompress_gbs"], 3),
            "same_payload_sizes": same, "ratio": round(comp_bytes / total, 5)}
    print(json.dumps(line), flush=True)
    codec.close()
    return 0 if plain["bit_exact"] and batched["bit_exact"] else 1


def run_sweep(args):
    """The sweep: 64 MiB of the text mix at block 18, level 5 (the file the reference's CPU codec runs as
    is), 1 GiB of lz_mix at block 16/18/20 x level 1/5/9, and 2 GiB of uniform random bytes at block
    16/18/20 (every block stored).  Per cell, device-resident: compress and decompress GB/s (CUDA
    events, mean of the timed steps), the ratio, the round trip bit-exact, and the first blocks' payloads
    compared byte for byte with the reference CPU codec's (oracle/_ref, when present)."""
    import numpy as np
    import torch
    import zero_cuda as Z
    import datagen as G
    ws, rank, local = dist_env()
    if rank != 0:
        return 0
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    have_ref = O.Ref.available()
    stream = torch.cuda.Stream(device=dev)
    sh = stream.cuda_stream
    cells = []
    plan = [("text_mix", 64 << 20, 18, 5)]  # the 64 MiB text mix the reference runs as-is on its CPU codec
    plan += [("lz_mix", args.size_mib << 20, bl, lv) for bl in (16, 18, 20) for lv in (1, 5, 9)]
    plan += [("random", 2 * (args.size_mib << 20), bl, 5) for bl in (16, 18, 20)]
    data_cache = {}
    with ClockSampler(local) as clk:
        for kind, n, bl, lv in plan:
            B = 1 << bl
            nb = (n + B - 1) // B
            key = (kind, n, bl)
            if key not in data_cache:
                data_cache.clear()
                data_cache[key] = (make_data(n, bl, 1000) if kind == "lz_mix" else G.text_mix(n, 7) if kind == "text_mix"
                                   else G.random_bytes(n, 77))
            host = data_cache[key]
            codec = Z.CudaCodec(level=lv, device=local)
            shape = None
            if args.autotune:  # the cell's launch shape chosen on a sample of its own data (no byte changes)
                shape = codec.autotune(host[:min(n, args.tune_mib << 20)], bl, lv)
            codec.prepare(bl)
            per = codec.batch_bytes(bl) // B
            dper = codec.batch_bytes_decode(bl) // B
            d_in = torch.zeros(n + 64, dtype=torch.uint8, device=dev)
            d_in[:n].copy_(torch.from_numpy(host))
            offs = torch.arange(nb, dtype=torch.int64, device=dev) * B
            lens = torch.clamp(n - offs, max=B).to(torch.int32)
            d_out = torch.zeros(n + 64, dtype=torch.uint8, device=dev)
            d_dec = torch.zeros(n + 64, dtype=torch.uint8, device=dev)
            methods = torch.zeros(nb, dtype=torch.uint8, device=dev)
            clens = torch.zeros(nb, dtype=torch.int32, device=dev)
            crcs = torch.zeros(nb, dtype=torch.int32, device=dev)
            dcrcs = torch.zeros(nb, dtype=torch.int32, device=dev)
            errs = torch.zeros(nb, dtype=torch.int32, device=dev)
            ooffs = torch.zeros(nb, dtype=torch.int64, device=dev)
            goffs = torch.zeros(nb, dtype=torch.int64, device=dev)
            chunks = [(b0, min(per, nb - b0)) for b0 in range(0, nb, per)]
            totals = torch.zeros(len(chunks), dtype=torch.int64, device=dev)
            base = torch.tensor([b0 * B for b0, k in chunks for _ in range(k)], dtype=torch.int64, device=dev)

            def compress():
                for ci, (b0, k) in enumerate(chunks):
                    o = b0 * B
                    codec.compress_device(d_in, offs[b0:], lens[b0:], k, bl, methods[b0:], clens[b0:], crcs[b0:],
                                          d_out[o:o + k * B + 64], ooffs[b0:], totals[ci:], stream=sh)
                with torch.cuda.stream(stream):
                    torch.add(ooffs, base, out=goffs)

            def decompress():
                for b0 in range(0, nb, dper):
                    k = min(dper, nb - b0)
                    codec.decompress_device(d_out, goffs[b0:], clens[b0:], methods[b0:], lens[b0:], k, bl, d_dec,
                                            offs[b0:], dcrcs[b0:], errs[b0:], stream=sh)

            for _ in range(args.warmup):
                compress()
                decompress()
            torch.cuda.synchronize(dev)
            ev = [_events(2) for _ in range(args.steps)]
            with torch.cuda.stream(stream):
                for i in range(args.steps):
                    ev[i][0][0].record(stream); compress(); ev[i][0][1].record(stream)
                    ev[i][1][0].record(stream); decompress(); ev[i][1][1].record(stream)
            torch.cuda.synchronize(dev)
            tc = sum(e[0][0].elapsed_time(e[0][1]) for e in ev) / args.steps
            td = sum(e[1][0].elapsed_time(e[1][1]) for e in ev) / args.steps
            ok = bool(torch.equal(d_dec[:n], d_in[:n])) and bool(torch.equal(dcrcs, crcs)) and not errs.any()
            comp = int(clens.sum().item())
            cell = {"data": kind, "bytes": n, "block_log": bl, "level": lv, "compress_gbs": round(n / tc / 1e6, 3),
                    "decompress_gbs": round(n / td / 1e6, 3), "round_trip_gbs": round(n / (tc + td) / 1e6, 3),
                    "ratio": round(comp / n, 5), "stored_blocks": int((methods == 0).sum().item()), "bit_exact": ok,
                    "shape": shape if shape is not None else codec.get_shape(bl, lv), "autotuned": shape is not None}
            if have_ref:
                k = min(nb, max(4, (8 << 20) >> bl))
                rm, rl, rp = O.Ref.cpu_compress(host[:k * B], bl, O.depth_for_level(lv))
                gm = methods[:k].cpu().numpy()
                gl = clens[:k].cpu().numpy()
                go = goffs[:k].cpu().numpy()
                span = d_out[:int(go[-1]) + int(gl[-1])].cpu().numpy()
                same = bool(np.array_equal(gm, np.asarray(rm, np.uint8)))
                for b in range(k):
                    if same and gm[b]:
                        same = span[int(go[b]):int(go[b]) + int(gl[b])].tobytes() == bytes(rp[b])
                cell["payloads_equal_reference"] = {"blocks": k, "equal": same}
                ok = ok and same
            cells.append(cell)
            print(json.dumps(cell), file=sys.stderr, flush=True)
            codec.close()
            del d_in, d_out, d_dec
            torch.cuda.empty_cache()
    head = next(c for c in cells if c["data"] == "lz_mix" and c["block_log"] == 18 and c["level"] == 5)
    all_ok = all(c["bit_exact"] and c.get("payloads_equal_reference", {"equal": True})["equal"] for c in cells)
    line = {"metric": METRIC, "value": head["round_trip_gbs"], "unit": "GB/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "dtype": "u8",
            "data": "synthetic (seeded lz_mix and uniform random generators)",
            "config": {"workload": f"sweep: text_mix 64 MiB at block 18 level 5; lz_mix {args.size_mib} MiB at "
                                   f"block 16/18/20 x level 1/5/9, random "
                                   f"{2 * args.size_mib} MiB at block 16/18/20 (level 5); value = the block 18 "
                                   f"level 5 cell's round trip",
                       "l2_flush": "none needed: every input is larger than the 126 MB L2"},
            "cells": cells, "bit_exact": all_ok, "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    return 0 if all_ok else 1


def run_archive(args):
    """Whole-archive workload: the many-file set of the batched config written as one .zero archive whose
    records, file CRCs (over each file's span, across blocks), entry table and footer are assembled on
    the GPU, then extracted with every block and file CRC checked.  value: the device-resident write
    (zc_archive_write_device), raw GB / CUDA-event time.  e2e: write + extract through the host-pointer
    calls (zc_archive_write, zc_archive_extract) with pinned buffers, copies included.  The reference's
    compress_archive (CPU codec, all host threads) writes a sample of the same files from the page cache,
    and the GPU writer's bytes for that sample must equal its archive."""
    import ctypes as C
    import shutil
    import tempfile
    import numpy as np
    import torch
    import zero_cuda as Z
    import datagen as G
    ws, rank, local = dist_env()
    if rank != 0:
        return 0
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    bl, level = args.block, args.level
    sizes, kinds = G.file_plan(args.files, 1 << 10, args.max_file_kib << 10, seed=2024)
    sizes = sizes.astype(np.int64)
    file_off = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
    total = int(sizes.sum())
    pinned = torch.zeros(total + 64, dtype=torch.uint8, pin_memory=True)
    hv = pinned.numpy()
    from concurrent.futures import ThreadPoolExecutor

    def gen(f):  # (the generators run in C without the interpreter lock: host threads fill files side by side)
        o, n = int(file_off[f]), int(sizes[f])
        k = int(kinds[f])
        out = hv[o:o + n]
        if k == 0:
            G.text_mix(n, 5000 + f, out=out)
        elif k == 1:
            G.lz_mix(n, bl, 5000 + f, out=out)
        else:
            G.random_bytes(n, 5000 + f, out=out)

    with ThreadPoolExecutor(16) as ex:
        list(ex.map(gen, range(args.files)))
    ext = ("txt", "lz", "rnd")
    entries = []
    for f in range(args.files):
        if f % 250 == 0:
            entries.append(Z.ArchiveEntry("d%03d" % (f // 250), 0, mtime=1700000000, is_dir=True))
        entries.append(Z.ArchiveEntry("d%03d/f%05d.%s" % (f // 250, f, ext[int(kinds[f])]), int(sizes[f]),
                                      mtime=1700000000 + f))
    ne = len(entries)
    L = Z.lib()
    arr, _keep = Z._c_entries(entries)
    cap = Z.archive_bound(entries, bl)
    codec = Z.CudaCodec(level=level, device=local)
    d_solid = torch.zeros(total + 64, dtype=torch.uint8, device=dev)
    d_solid.copy_(pinned)
    d_out = torch.zeros(cap, dtype=torch.uint8, device=dev)
    d_len = torch.zeros(1, dtype=torch.int64, device=dev)
    d_ecrc = torch.zeros(ne, dtype=torch.int32, device=dev)
    stream = torch.cuda.Stream(device=dev)
    sh = stream.cuda_stream

    def check(rc):
        if rc:
            Z._raise(codec._ctx, rc)

    def write_dev():
        check(L.zc_archive_write_device(codec._ctx, d_solid.data_ptr(), bl, level, arr, ne, d_out.data_ptr(), cap,
                                        d_len.data_ptr(), d_ecrc.data_ptr(), sh))

    for _ in range(args.warmup):
        write_dev()
    torch.cuda.synchronize(dev)
    ev = _events(args.steps)
    l0 = codec.launch_count()
    with ClockSampler(local) as clk:
        with torch.cuda.stream(stream):
            for i in range(args.steps):
                ev[i][0].record(stream)
                write_dev()
                ev[i][1].record(stream)
        torch.cuda.synchronize(dev)
    t_w = sum(a.elapsed_time(b) for a, b in ev) / args.steps
    launches = (codec.launch_count() - l0) // args.steps
    alen = int(d_len.item())
    dev_arch = d_out[:alen].cpu().numpy()
    codec.profile(True)
    write_dev()
    torch.cuda.synchronize(dev)
    stages = codec.profile_stages()
    codec.profile(False)
    # e2e: the host-pointer write and extract, pinned buffers
    h_arch = torch.zeros(cap, dtype=torch.uint8, pin_memory=True).numpy()
    h_back = torch.zeros(total + 64, dtype=torch.uint8, pin_memory=True).numpy()
    out_len = C.c_uint64()

    def e2e_step():
        check(L.zc_archive_write(codec._ctx, hv.ctypes.data, bl, level, arr, ne, h_arch.ctypes.data, cap,
                                 C.byref(out_len)))
        check(L.zc_archive_extract(codec._ctx, h_arch.ctypes.data, out_len.value, h_back.ctypes.data, total))

    e2e_step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    t_e = (time.perf_counter() - t0) / args.steps
    ok = (out_len.value == alen and np.array_equal(h_arch[:alen], dev_arch)
          and np.array_equal(h_back[:total], hv[:total])
          and [int(x) & 0xFFFFFFFF for x in d_ecrc.cpu().tolist()] == [int(arr[i].crc) for i in range(ne)])
    info, _ = Z.read_table(dev_arch)
    # the dominant kernel of one (profiled) write; algorithmic bytes of a write: raw read + archive written
    peak, peak_kind = peaks()
    dom_name, (dom_ms, dom_n) = max(stages.items(), key=lambda kv: kv[1][0])
    alg = total + alen
    roof = {"bound": "hbm", "kernel": dom_name, "achieved": round(alg / (dom_ms * 1e-3) / GB, 2), "peak": peak,
            "unit": "GB/s", "frac": round(alg / (dom_ms * 1e-3) / GB / peak, 4), "traffic": None,
            "peak_source": peak_kind, "algorithmic_bytes_per_launch": int(alg / max(1, dom_n)),
            "avg_launch_ms": round(dom_ms / max(1, dom_n), 4),
            "pipeline_frac": round(alg / (t_w * 1e-3) / GB / peak, 4)}
    line = {"metric": METRIC, "value": round(total / t_w / 1e6, 3), "unit": "GB/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(t_w, 3), "higher_is_better": True,
            "scaling": "weak", "dtype": "u8", "data": "synthetic (seeded per-file generators)",
            "config": {"workload": f"archive: {args.files} files in {ne - args.files} folders, sizes log-uniform "
                                   f"1 KiB-{args.max_file_kib} KiB ({total / 2**30:.2f} GiB), generators "
                                   f"text/lz/random, block {bl}, level {level}: the whole .zero archive written on "
                                   f"the GPU (records, file CRCs, table, footer)",
                       "blocks": int(info["n_blocks"]), "bytes": total, "archive_bytes": alen,
                       "l2_flush": "none needed: input larger than the 126 MB L2"},
            "ratio": round(alen / total, 5), "bit_exact": bool(ok), "gpu_launches": launches, "roofline": roof,
            "stages_ms_per_step": {k: round(v[0], 4) for k, v in stages.items()},
            "e2e": {"value": round(total / t_e / 1e9, 4), "unit": "GB/s",
                    "h2d_bytes_per_step": int(total + alen), "d2h_bytes_per_step": int(alen + total),
                    "path": "zc_archive_write + zc_archive_extract (every block and file CRC checked), pinned "
                            "host buffers"},
            "clocks": clk.summary()}
    if not args.no_cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        if O.Ref.available():
            base = "/dev/shm" if os.path.isdir("/dev/shm") else None
            tmp = tempfile.mkdtemp(prefix="zc_arch_", dir=base)
            try:
                root = os.path.join(tmp, "data")
                picked = 0
                for e in entries:
                    p = os.path.join(root, e.name)
                    if e.is_dir:
                        os.makedirs(p, exist_ok=True)
                        continue
                    if picked >= (256 << 20):
                        break
                    f = int(e.name.split("/f")[1].split(".")[0])
                    with open(p, "wb") as fh:
                        fh.write(hv[int(file_off[f]):int(file_off[f]) + e.size].tobytes())
                    picked += e.size
                for dp, dn, fn in os.walk(root):
                    for x in dn + fn:
                        os.utime(os.path.join(dp, x), (1700000000, 1700000000))
                os.utime(root, (1700000000, 1700000000))
                zpath = os.path.join(tmp, "ref.zero")
                t0 = time.perf_counter()
                O.Ref.compress_archive([root], zpath, block_log=bl, level=level)
                t_ref = time.perf_counter() - t0
                with open(zpath, "rb") as fh:
                    ref = fh.read()
                _, rents = Z.read_table(ref)
                solid = b"".join(open(os.path.join(tmp, e.name), "rb").read() for e in rents if not e.is_dir)
                same = codec.archive_write(solid, rents, bl, level=level) == ref
                line["cpu_baseline"] = {"value": round(picked / t_ref / 1e9, 4), "unit": "GB/s",
                                        "cores": O.Ref.hardware_threads(), "kind": "reference",
                                        "sample": f"compress_archive of the first {picked >> 20} MiB of the files "
                                                  f"(page cache), CPU codec, block {1 << bl >> 10} KiB, level {level}"}
                line["same_as_reference_archive"] = bool(same)
                ok = ok and same
            finally:
                shutil.rmtree(tmp, ignore_errors=True)
    line["bit_exact"] = bool(ok)
    print(json.dumps(line), flush=True)
    codec.close()
    return 0 if ok else 1


def reference_archive(hv, bl, level):
    """The CPU-baseline leg of the decode workload: the reference CPU codec (compiled from the reference's
    sources, all host threads) writes the archive's records for the whole input, timed.  Returns
    (methods, comp_lens, bodies blob, body offsets, seconds, threads), or None without the compiled
    reference."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import oracle as O
    if not O.Ref.available():
        return None
    B = 1 << bl
    t0 = time.perf_counter()
    methods, lens, pays = O.Ref.cpu_compress(hv, bl, O.depth_for_level(level))
    dt = time.perf_counter() - t0
    nb = len(methods)
    clens = np.array([int(lens[b]) if methods[b] else min(B, hv.size - b * B) for b in range(nb)], np.int64)
    coffs = np.concatenate([[0], np.cumsum(clens)[:-1]]).astype(np.int64)
    blob = np.empty(int(clens.sum()) + 64, np.uint8)
    for b in range(nb):
        o = int(coffs[b])
        if methods[b]:
            blob[o:o + int(clens[b])] = np.frombuffer(pays[b], np.uint8)
        else:
            blob[o:o + int(clens[b])] = hv[b * B:b * B + int(clens[b])]
    del pays
    return methods.copy(), clens, blob, coffs, dt, O.Ref.hardware_threads()


def run_decode(args):
    """Decode-heavy workload (the decode config): LZ-mix data at block 2^20, level 9.  The archive's records
    are written by the reference CPU codec (the CPU-baseline leg, timed on the host's threads; without the
    compiled reference, by the GPU encoder) and also by the GPU encoder, whose payloads must equal the
    reference's for every block; then the reference-written records are extracted K times on the GPU.
    Each extract decodes every block and computes its CRC-32 (test = the same plus the comparison)."""
    import numpy as np
    import torch
    import zero_cuda as Z
    import datagen as G
    from concurrent.futures import ThreadPoolExecutor
    ws, rank, local = dist_env()
    if rank != 0:
        return 0
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    bl, level = args.block, args.level
    B = 1 << bl
    n = args.size_mib << 20
    nb = (n + B - 1) // B
    pinned = torch.empty(n, dtype=torch.uint8, pin_memory=True)
    hv = pinned.numpy()
    piece = 256 << 20  # generated in pieces of 256 MiB, one seed each, on host threads
    with ThreadPoolExecutor(8) as ex:
        list(ex.map(lambda i: G.lz_mix(min(piece, n - i * piece), bl, 7000 + i, out=hv[i * piece:i * piece + min(piece, n - i * piece)]),
                    range((n + piece - 1) // piece)))
    codec = Z.CudaCodec(level=level, device=local)
    d_in = torch.zeros(n + 64, dtype=torch.uint8, device=dev)
    d_in[:n].copy_(pinned)
    offs = torch.arange(nb, dtype=torch.int64, device=dev) * B
    lens = torch.clamp(n - offs, max=B).to(torch.int32)
    d_out = torch.zeros(n + 64, dtype=torch.uint8, device=dev)
    d_dec = torch.zeros(n + 64, dtype=torch.uint8, device=dev)
    methods = torch.zeros(nb, dtype=torch.uint8, device=dev)
    clens = torch.zeros(nb, dtype=torch.int32, device=dev)
    crcs = torch.zeros(nb, dtype=torch.int32, device=dev)
    dcrcs = torch.zeros(nb, dtype=torch.int32, device=dev)
    errs = torch.zeros(nb, dtype=torch.int32, device=dev)
    ooffs = torch.zeros(nb, dtype=torch.int64, device=dev)
    goffs = torch.zeros(nb, dtype=torch.int64, device=dev)
    per = codec.batch_bytes(bl) // B
    chunks = [(b0, min(per, nb - b0)) for b0 in range(0, nb, per)]
    totals = torch.zeros(len(chunks) + 1, dtype=torch.int64, device=dev)
    stream = torch.cuda.Stream(device=dev)
    sh = stream.cuda_stream
    t0 = time.perf_counter()
    for ci, (b0, k) in enumerate(chunks):
        o = b0 * B
        codec.compress_device(d_in, offs[b0:], lens[b0:], k, bl, methods[b0:], clens[b0:], crcs[b0:],
                              d_out[o:o + k * B + 64], ooffs[b0:], totals[ci:], stream=sh)
    chunk_base = torch.tensor([b0 * B for b0, k in chunks for _ in range(k)], dtype=torch.int64, device=dev)
    with torch.cuda.stream(stream):
        torch.add(ooffs, chunk_base, out=goffs)
    torch.cuda.synchronize(dev)
    t_comp = time.perf_counter() - t0
    comp = int(clens.sum().item())
    dper = codec.batch_bytes_decode(bl) // B
    writer, same, cpu = "GPU encoder", None, None
    ref = None if args.no_cpu else reference_archive(hv, bl, level)
    if ref is not None:
        r_meth, r_clens, r_blob, r_coffs, r_dt, r_thr = ref
        # the GPU encoder's records against the reference's, every block
        g_meth = methods.cpu().numpy()
        g_clens = clens.cpu().numpy().astype(np.int64)
        g_offs = goffs.cpu().numpy()
        same = bool(np.array_equal(g_meth, r_meth))
        if same:
            host_out = d_out.cpu().numpy()
            for b in range(nb):
                if r_meth[b] and (g_clens[b] != r_clens[b] or not np.array_equal(
                        host_out[g_offs[b]:g_offs[b] + g_clens[b]], r_blob[r_coffs[b]:r_coffs[b] + r_clens[b]])):
                    same = False
                    break
            del host_out
        # the extract below decodes the reference-written records
        d_out = torch.from_numpy(r_blob).to(dev)
        goffs = torch.from_numpy(r_coffs).to(dev)
        clens = torch.from_numpy(r_clens.astype(np.int32)).to(dev)
        methods = torch.from_numpy(r_meth.astype(np.uint8)).to(dev)
        comp = int(r_clens.sum())
        writer = "reference CPU codec (oracle/_ref, the reference's own sources)"
        cpu = {"value": round(n / r_dt / GB, 4), "unit": "GB/s", "cores": r_thr, "kind": "reference",
               "sample": f"the whole {args.size_mib} MiB compressed at block {bl}, level {level} (the archive the "
                         "GPU extracts)"}
        del r_blob

    def decompress():
        for b0 in range(0, nb, dper):
            k = min(dper, nb - b0)
            codec.decompress_device(d_out, goffs[b0:], clens[b0:], methods[b0:], lens[b0:], k, bl, d_dec, offs[b0:],
                                    dcrcs[b0:], errs[b0:], stream=sh)

    if args.fill_words or args.fill_ring_log or args.fill_warps:
        kw = {k: v for k, v in (("fill_words", args.fill_words), ("fill_ring_log", args.fill_ring_log),
                                ("fill_warps", args.fill_warps)) if v}
        codec.set_shape(bl, level, **kw)
    codec.prepare(bl)
    codec.set_graphs(True)
    for _ in range(args.warmup):
        decompress()
    torch.cuda.synchronize(dev)
    ev = _events(args.steps)
    l0 = codec.launch_count()
    with ClockSampler(local) as clk:
        with torch.cuda.stream(stream):
            for i in range(args.steps):
                ev[i][0].record(stream); decompress(); ev[i][1].record(stream)
        torch.cuda.synchronize(dev)
    launches = codec.launch_count() - l0
    t = sum(a.elapsed_time(b) for a, b in ev) / args.steps
    # per-kernel times: graph replays carry no per-stage events, so the same steps once more without them
    codec.set_graphs(False)
    codec.profile(True)
    with torch.cuda.stream(stream):
        for i in range(args.steps):
            decompress()
    torch.cuda.synchronize(dev)
    stages = codec.profile_stages()
    codec.profile(False)
    ok = bool(torch.equal(d_dec[:n], d_in[:n])) and bool(torch.equal(dcrcs, crcs)) and not errs.any()
    peak, _ = peaks()
    dom = max(stages.items(), key=lambda kv: kv[1][0]) if stages else ("", (0.0, 1))
    per_launch = (n + comp) / max(1, dom[1][1] // max(1, args.steps))
    achieved = (n + comp) * args.steps / (dom[1][0] * 1e-3) / GB if dom[1][0] else 0.0
    line = {"metric": METRIC, "value": round(n / (t * 1e-3) / GB, 4), "unit": "GB/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(t, 4), "higher_is_better": True,
            "scaling": "weak", "dtype": "u8", "data": "synthetic (seeded lz_mix generator, 256 MiB pieces)",
            "config": {"workload": f"decode-heavy: lz_mix {args.size_mib} MiB, block {bl}, level {level}: "
                                   "extract (decode + CRC-32 of every block)", "blocks": nb,
                       "l2_flush": "none needed: input larger than the 126 MB L2"},
            "ratio": round(comp / n, 5), "bit_exact": ok, "compress_s_untimed": round(t_comp, 3),
            "roofline": {"bound": "hbm", "kernel": dom[0], "achieved": round(achieved, 2), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "algorithmic_bytes_per_launch": int(per_launch),
                         "traffic": (int(DRAM_BYTES_PER_RAW_BYTE[dom[0]] * n / max(1, dom[1][1] // max(1, args.steps)))
                                     if dom[0] in DRAM_BYTES_PER_RAW_BYTE else None),
                         "pipeline_frac": round((n + comp) / (t * 1e-3) / GB / peak, 4)},
            "stages_ms_per_step": {k: round(v[0] / args.steps, 4) for k, v in stages.items()},
            "gpu_launches": int(launches), "clocks": clk.summary(), "fill_shape": codec.get_shape(bl, level),
            "archive_written_by": writer, "payloads_equal_reference_all_blocks": same}
    if cpu is not None:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)
    codec.close()
    return 0 if ok else 1


def pinned_copy(a):
    """(numpy view, owning tensor) of a page-locked copy of u8 array a."""
    import torch
    t = torch.empty(max(a.size, 1), dtype=torch.uint8, pin_memory=True)
    v = t.numpy()[:a.size]
    v[:] = a
    return v, t


def run_serve(args):
    """The serving workload: an open-loop Poisson stream of jobs (60 % compress, 30 % extract, 10 % test),
    each one file of log-uniform size from the many-file generator mix, block size from {16, 18, 20}, level
    from {1, 5, 9}, under a device-memory admission budget.  The arrival rate is swept upward until the
    server saturates; per rate: p50 / p99 latency (submission to completion) and aggregate GB/s."""
    import threading
    import queue
    import numpy as np
    import zero_cuda as Z
    import datagen as G
    ws, rank, local = dist_env()
    if rank != 0:
        return 0
    rng = np.random.default_rng(4242)
    pool = []
    sizes, kinds = G.file_plan(args.pool, 4 << 10, args.max_job_mib << 20, seed=4242)
    with Z.CudaCodec(level=5, device=local) as codec:
        for i in range(args.pool):
            bl = int(rng.choice([16, 18, 20]))
            lv = int(rng.choice([1, 5, 9]))
            data = G.by_kind(int(kinds[i]), int(sizes[i]), bl, 8000 + i)
            meth, lens, crcs, pay, offs = codec.compress_arrays(data, bl, level=lv)
            blob, clens, rlens = Z.record_bodies(data, meth, lens, pay, offs, bl)
            # the clients' buffers are page-locked, as a server's I/O buffers would be
            pdata, pblob = pinned_copy(data), pinned_copy(blob)
            pool.append(dict(data=pdata[0], bl=bl, lv=lv, blob=pblob[0], clens=clens, meth=meth.copy(), rlens=rlens,
                             crcs=crcs.copy(), keep=(pdata[1], pblob[1])))
    srv = Z.Server(budget_bytes=args.budget_gib << 30, device=local, pinned=True)
    plain_codec = Z.CudaCodec(level=5, device=local)
    rates = [float(r) for r in args.rates.split(",")]
    results = []

    def draw_jobs(rate):
        """The job stream of one rate: (arrival s, pool index, kind u), from the rate's own seed, so that the
        served and the plain form see the same jobs at the same times."""
        g = np.random.default_rng(int(rate * 1000) + 17)
        out, t = [], 0.0
        while True:
            t += g.exponential(1.0 / rate)
            if t > args.duration:
                return out
            out.append((t, int(g.integers(len(pool))), float(g.random())))

    def plain_form(jobs):
        """The plain per-job form: one worker takes the jobs in arrival order and runs each alone through the
        host-pointer calls (zc_compress; zc_decompress, CRCs compared for a test), as a server without
        batching would."""
        q = queue.Queue()
        lat, nb = [], [0]

        def worker():
            while True:
                item = q.get()
                if item is None:
                    return
                t_arr, idx, u = item
                j = pool[idx]
                if u < 0.6:
                    plain_codec.compress_arrays(j["data"], j["bl"], level=j["lv"])
                    nb[0] += j["data"].size
                else:
                    coffs = np.concatenate([[0], np.cumsum(j["clens"])[:-1]]).astype(np.uint64)
                    plain_codec.prepare(j["bl"])
                    raw, crcs, errs = plain_codec.decompress_arrays(j["blob"], coffs, j["clens"], j["meth"], j["rlens"])
                    if u >= 0.9:
                        assert np.array_equal(crcs, j["crcs"])
                    nb[0] += int(j["rlens"].sum())
                lat.append(time.perf_counter() - (t0p + t_arr))

        th = threading.Thread(target=worker, daemon=True)
        t0p = time.perf_counter()
        th.start()
        for t_arr, idx, u in jobs:
            delay = t0p + t_arr - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            q.put((t_arr, idx, u))
        q.put(None)
        th.join()
        wall = time.perf_counter() - t0p
        lat_ms = np.array(lat) * 1e3
        return {"achieved_gbs": round(nb[0] / wall / 1e9, 3), "wall_s": round(wall, 2),
                "p50_ms": round(float(np.percentile(lat_ms, 50)), 2) if len(lat) else None,
                "p99_ms": round(float(np.percentile(lat_ms, 99)), 2) if len(lat) else None}

    for rate in rates:
        jobs = draw_jobs(rate)
        done_q = queue.Queue()
        lat, nbytes, statuses = [], [0], []

        def waiter():
            while True:
                h = done_q.get()
                if h is None:
                    return
                srv.wait(h, raise_on_error=False)
                lat.append(h.latency)
                statuses.append(h.status)
                nbytes[0] += h.nbytes

        th = threading.Thread(target=waiter, daemon=True)
        th.start()
        t0 = time.perf_counter()
        t_next = 0.0
        njobs = 0
        s0 = srv.stats()
        for t_next, idx, u in jobs:
            delay = t0 + t_next - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            j = pool[idx]
            if u < 0.6:
                h = srv.compress(j["data"], j["bl"], j["lv"])
                h.nbytes = j["data"].size
            elif u < 0.9:
                h = srv.extract(j["blob"], j["clens"], j["meth"], j["rlens"], j["bl"])
                h.nbytes = int(j["rlens"].sum())
            else:
                h = srv.test(j["blob"], j["clens"], j["meth"], j["rlens"], j["crcs"], j["bl"])
                h.nbytes = int(j["rlens"].sum())
            done_q.put(h)
            njobs += 1
        done_q.put(None)
        th.join()
        wall = time.perf_counter() - t0
        s1 = srv.stats()
        lat_ms = np.array(lat) * 1e3
        results.append({"rate_jobs_per_s": rate, "jobs": njobs, "offered_gbs": round(nbytes[0] / args.duration / 1e9, 3),
                        "achieved_gbs": round(nbytes[0] / wall / 1e9, 3),
                        "p50_ms": round(float(np.percentile(lat_ms, 50)), 2) if njobs else None,
                        "p99_ms": round(float(np.percentile(lat_ms, 99)), 2) if njobs else None,
                        "ticks": s1["ticks"] - s0["ticks"], "errors": int(sum(1 for x in statuses if x)),
                        "wall_s": round(wall, 2),
                        "gpu_busy": round((s1["gpu_s"] - s0["gpu_s"]) / wall, 3),
                        "worker_s": {k: round(s1[k] - s0[k], 3) for k in ("wait_s", "handout_s", "upload_s")}})
        if not args.no_plain:
            results[-1]["plain"] = plain_form(jobs)
        print(json.dumps({"serve_rate": results[-1]}), file=sys.stderr, flush=True)
        if wall > args.duration * 2.0:  # saturated: the backlog took as long again as the arrivals
            break
    srv.close()
    plain_codec.close()
    best = max(results, key=lambda r: r["achieved_gbs"])
    line = {"metric": METRIC, "value": best["achieved_gbs"], "unit": "GB/s", "n_gpus": 1, "higher_is_better": True,
            "scaling": "weak", "dtype": "u8", "data": "synthetic (seeded per-file generators)",
            "config": {"workload": f"serving: Poisson jobs 60/30/10 compress/extract/test, sizes log-uniform "
                                   f"4 KiB-{args.max_job_mib} MiB (pool of {args.pool} files), block 16/18/20, "
                                   f"level 1/5/9, {args.budget_gib} GiB admission budget, {args.duration} s per rate"},
            "p50_ms": best["p50_ms"], "p99_ms": best["p99_ms"], "plain_at_that_rate": best.get("plain"),
            "plain_best_gbs": max((r["plain"]["achieved_gbs"] for r in results if "plain" in r), default=None),
            "sweep": results}
    print(json.dumps(line), flush=True)
    return 0 if all(r["errors"] == 0 for r in results) else 1


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--block", type=int, default=None, help="default 18; 20 for --config decode")
    ap.add_argument("--level", type=int, default=None, help="default 5; 9 for --config decode")
    ap.add_argument("--size-mib", type=int, default=None, help="default 1024; 8192 for --config decode")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--config", choices=["lz", "batched", "decode", "serve", "archive", "sweep"], default="lz",
                    help="lz: the headline round trip; batched: many files, plain vs batched; decode: extract-heavy; "
                         "serve: the request loop; archive: whole .zero archives of many files; sweep: lz_mix at "
                         "block 16/18/20 x level 1/5/9 and random bytes")
    ap.add_argument("--fill-words", type=int, default=0, help="decode: the fill's words a lane a round (1, 2, 4)")
    ap.add_argument("--fill-ring-log", type=int, default=0, help="decode: the fill's ring size (log2 bytes)")
    ap.add_argument("--fill-warps", type=int, default=0, help="decode: the fill's warps per CTA")
    ap.add_argument("--chunk-mib", type=int, default=0, help="batched: encoder launches of at most this many MiB")
    ap.add_argument("--no-plain", action="store_true", help="serve: skip the plain per-job form beside the server")
    ap.add_argument("--autotune", action="store_true", help="sweep: autotune each cell's launch shape first")
    ap.add_argument("--tune-mib", type=int, default=128, help="sweep: the autotuner's sample of each cell (MiB)")
    ap.add_argument("--files", type=int, default=10000)
    ap.add_argument("--max-file-kib", type=int, default=1024)
    ap.add_argument("--pool", type=int, default=48, help="serve: distinct files the jobs draw from")
    ap.add_argument("--max-job-mib", type=int, default=256, help="serve: the largest job")
    ap.add_argument("--budget-gib", type=int, default=112, help="serve: device memory admission budget (GiB)")
    ap.add_argument("--rates", default="8,32,64,128,256,512", help="serve: arrival rates to sweep (jobs/s)")
    ap.add_argument("--duration", type=float, default=6.0, help="serve: seconds of arrivals per rate")
    args = ap.parse_args()
    dec = args.config == "decode"  # the decode-heavy workload: an 8 GiB archive at block 20, level 9
    if args.block is None:
        args.block = 20 if dec else 18
    if args.level is None:
        args.level = 9 if dec else 5
    if args.size_mib is None:
        args.size_mib = 8192 if dec else 1024
    if args.impl == "reference":
        return run_reference(args)
    if args.config == "batched":
        return run_batched(args)
    if args.config == "decode":
        return run_decode(args)
    if args.config == "serve":
        return run_serve(args)
    if args.config == "archive":
        return run_archive(args)
    if args.config == "sweep":
        return run_sweep(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
