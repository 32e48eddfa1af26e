"""Autotuner for the scalar strided-batch solves.

Sweeps, on the current GPU, every algorithm the dispatcher offers for each
(dtype, axis class, system length) bucket and writes the winners as a tuning
table that the C ABI reads (``tridLoadTuningTable`` or the environment
variable ``TRID_B200_TUNING``).

    python -m tridsolver_b200.autotune --out tuning_b200.txt [--dtypes f64,f32]
                                       [--lengths 32,64,128,256,512] [--elems 16777216]

Candidates (see tridSetMethod in include/trid_b200.h):
    method 1            Thomas, one thread per system, c'/d' in scratch
    method 2/3, chunk   partitioned Thomas with warp PCR (2 = TMA staging
                        when possible, 3 = plain loads), with every
                        rows-per-thread chunk that covers n and, on strided
                        axes, 4/8/16 systems per CTA (and 32 for method 2;
                        128 bytes of systems, 16 FP64 / 32 FP32, is the
                        streamed persistent kernel)
    method 6, chunk     axis 0, longer systems: one CTA per system, 4/8/16
                        rows per thread (up to 4096 rows)
    (method 2 above 512 rows on axis 0 also means the blocked partition:
    block reduction, recursive block solve, block finish; its chunk 8 or 16
    is the block size, 256 or 512 rows, swept for lengths past 4096)

Axis class 4 is the variable-length batch: its length buckets (2 rows per
lane up to m2max rows, 4 up to m4max, else 8) are swept on a batch of short
systems (lengths log-uniform on [8, 256]) and written as class-4 lines.

--stride-sweep instead times the default algorithm on FP64 problems of
64 M unknowns whose solve axis has plane strides from 8 KiB to 2 MiB, against
the streamed full-line tiles and the narrow (8 and 16 system) plain and
TMA-staged tiles: 64-byte row segments lose much of DRAM's rate once the
stride reaches 64 KiB.

Axis classes: 0 = solve along axis 0 (unit stride); 1 = strided, row stride
<= 64 KiB; 2 = <= 1 MiB; 3 = larger strides (swept with --classes 0,1,2,3).
The timing problem of each bucket holds about ``--elems`` unknowns (16.7 M by
default, > L2 for FP64 and FP32) shaped as [n, S] (class 0), [256, n, S]
(class 1) or [256, S, n] (class 2); class 3 uses [32, S, n] with S >= 8192
(a 2 MiB row stride in FP64).
"""

import argparse
import ctypes
import json
import sys

import numpy as np

from ._lib import TridError, lib

CHUNKS = (2, 4, 8, 16)


def need_chunk(n):
    for ch in CHUNKS:
        if n <= 32 * ch:
            return ch
    return 0


def candidates(axis, n):
    out = [(1, 0, 0)]
    ch0 = need_chunk(n)
    if ch0:
        for ch in CHUNKS:
            if ch < ch0:
                continue
            if axis == 0:
                out.append((2, ch, 0))
                out.append((3, ch, 0))
            else:
                for spc in (4, 8, 16):
                    out.append((2, ch, spc))
                    out.append((3, ch, spc))
                out.append((2, ch, 32))
    if axis == 0 and n > 64:
        if n <= 4096:
            for ch in (4, 8, 16):
                out.append((6, ch, 0))
        if not ch0:
            out.append((2, 8, 0))   # blocked partition, 256-row blocks
            out.append((2, 16, 0))  # 512-row blocks
    if axis > 0 and not ch0:
        # strided systems past 512 rows: the blocked partition, 256- or
        # 512-row blocks, 8 or 16 systems per CTA
        for ch in (8, 16):
            for spc in (8, 16):
                out.append((2, ch, spc))
    return out


# (m2max, m4max) settings of the variable-length buckets
VARLEN_BUCKETS = ((64, 128), (32, 128), (0, 128), (64, 64), (32, 64), (0, 0))


def varlen_entries(dt, m2max, m4max):
    """Class-4 table lines for the bucket cut-offs (m2max, m4max)."""
    out = []
    if m2max:
        out.append((dt, 4, m2max, (2, 2, 0)))
    if m4max > m2max:
        out.append((dt, 4, m4max, (2, 4, 0)))
    out.append((dt, 4, 256, (2, 8, 0)))
    return out


def tune_varlen(dt, nsys=400_000, reps=10, verbose=True, seed=3):
    """Time every bucket setting on one batch of short systems; returns the
    winning table lines and the timings."""
    import os
    import tempfile

    import torch

    from .varlen import solve_varlen

    tdtype = torch.float64 if dt == "f64" else torch.float32
    rng = np.random.default_rng(seed)
    lens = np.floor(np.exp(rng.uniform(np.log(8), np.log(256), nsys))).astype(np.int64)
    off = torch.from_numpy(np.concatenate([[0], np.cumsum(lens)])).cuda()
    total = int(lens.sum())
    g = torch.Generator(device="cuda").manual_seed(seed)
    a = torch.rand(total, device="cuda", dtype=tdtype, generator=g) * 2 - 1
    c = torch.rand(total, device="cuda", dtype=tdtype, generator=g) * 2 - 1
    b = a.abs() + c.abs() + 1 + torch.rand(total, device="cuda", dtype=tdtype, generator=g)
    d = torch.randn(total, device="cuda", dtype=tdtype, generator=g)
    L = lib()
    report, best = [], None
    fd, path = tempfile.mkstemp(suffix=".txt")
    os.close(fd)
    try:
        for m2, m4 in VARLEN_BUCKETS:
            entries = varlen_entries(dt, m2, m4)
            write_table(entries, path)
            if L.tridLoadTuningTable(path.encode()) != 0:
                raise TridError(3, "tridLoadTuningTable")
            x = d.clone()
            for _ in range(3):
                solve_varlen(a, b, c, x, off, total)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(reps):
                solve_varlen(a, b, c, x, off, total)
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / reps
            gbs = (5 * tdtype.itemsize * total + 8 * (nsys + 1)) / (ms * 1e-3) / 1e9
            report.append({"dtype": dt, "axis": 4, "m2max": m2, "m4max": m4, "ms": ms,
                           "GBs": round(gbs, 1)})
            if verbose:
                print(f"{dt} varlen m2max={m2:3d} m4max={m4:3d}: {ms:.4f} ms {gbs:8.1f} GB/s",
                      file=sys.stderr)
            if best is None or ms < best[0]:
                best = (ms, entries)
    finally:
        L.tridLoadTuningTable(None)
        os.unlink(path)
    return best[1], report


def problem_dims(axis, n, elems):
    if axis == 0:
        return [n, max(1, elems // n)], 0
    if axis == 3:
        return [32, max(8192, elems // (32 * n)), n], 2
    rest = max(1, elems // (256 * n))
    if axis == 1:
        return [256, n, rest], 1
    return [256, rest, n], 2


def time_candidate(torch, dtype, dims, solvedim, method, reps=10):
    L = lib()
    size = int(np.prod(dims))
    g = torch.Generator(device="cuda").manual_seed(7)
    a = torch.rand(size, device="cuda", dtype=dtype, generator=g) * 2 - 1
    c = torch.rand(size, device="cuda", dtype=dtype, generator=g) * 2 - 1
    b = a.abs() + c.abs() + 1 + torch.rand(size, device="cuda", dtype=dtype, generator=g)
    d = torch.randn(size, device="cuda", dtype=dtype, generator=g)
    fn = L.tridDmtsvStridedBatch if dtype == torch.float64 else L.tridSmtsvStridedBatch
    dims_c = (ctypes.c_int * len(dims))(*dims)
    st = L.tridSetMethod(*method)
    if st != 0:
        raise TridError(st, "tridSetMethod")
    L.tridSetStream(ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    args = [ctypes.c_void_p(t.data_ptr()) for t in (a, b, c, d)] + [None, len(dims), solvedim,
                                                                     dims_c, dims_c]
    try:
        for _ in range(3):
            st = fn(*args)
            if st != 0:
                raise TridError(st, "solve")
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn(*args)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps
    finally:
        L.tridSetMethod(0, 0, 0)


def tune(dtypes=("f64", "f32"), lengths=(32, 64, 128, 256, 512), elems=1 << 24, verbose=True,
         classes=(0, 1, 2)):
    import torch

    table, report = [], []
    for dt in dtypes:
        tdtype = torch.float64 if dt == "f64" else torch.float32
        for axis in classes:
            if axis == 4:
                entries, rep = tune_varlen(dt, verbose=verbose)
                table.extend((e[0], e[1], e[2], e[3]) for e in entries)
                report.extend(rep)
                continue
            for n in lengths:
                dims, sd = problem_dims(axis, n, elems)
                best = None
                # the built-in choice, for comparison (not a table candidate)
                ms = time_candidate(torch, tdtype, dims, sd, (0, 0, 0))
                report.append({"dtype": dt, "axis": axis, "n": n, "method": "built-in", "ms": ms,
                               "GBs": round(5 * tdtype.itemsize * int(np.prod(dims)) /
                                            (ms * 1e-3) / 1e9, 1)})
                for m in candidates(axis, n):
                    ms = time_candidate(torch, tdtype, dims, sd, m)
                    gbs = 5 * tdtype.itemsize * int(np.prod(dims)) / (ms * 1e-3) / 1e9
                    report.append({"dtype": dt, "axis": axis, "n": n, "method": m, "ms": ms,
                                   "GBs": round(gbs, 1)})
                    if verbose:
                        print(f"{dt} axis{axis} n={n:5d} method={m}: {ms:.4f} ms {gbs:8.1f} GB/s",
                              file=sys.stderr)
                    if best is None or ms < best[0]:
                        best = (ms, m)
                table.append((dt, axis, n, best[1]))
    return table, report


STRIDE_SHAPES = (([256, 4, 256, 256], 2), ([256, 16, 256, 64], 2), ([256, 256, 256], 1),
                 ([256, 256, 256], 2), ([1024, 64, 256], 2), ([2048, 128, 256], 2))


def stride_sweep(methods=((0, 0, 0), (2, 8, 16), (2, 8, 8), (3, 8, 8), (3, 8, 16))):
    """GB/s of FP64 solves of n=256 on strided axes whose plane stride grows
    from 8 KiB to 2 MiB (the same 40 B/unknown and about 64 M unknowns each)."""
    import torch

    out = []
    for m in methods:
        for dims, sd in STRIDE_SHAPES:
            ms = time_candidate(torch, torch.float64, dims, sd, m)
            size = int(np.prod(dims))
            row = {"dims": dims, "solvedim": sd, "method": list(m),
                   "plane_stride_kib": int(np.prod(dims[:sd])) * 8 // 1024,
                   "GBs": round(40 * size / (ms * 1e-3) / 1e9, 1)}
            print(json.dumps(row), flush=True)
            out.append(row)
            torch.cuda.empty_cache()
    return out


def write_table(table, path):
    with open(path, "w") as f:
        f.write("# dtype axis_class nmax method chunk sys_per_cta (tridsolver_b200.autotune)\n")
        for dt, axis, n, (m, ch, spc) in table:
            f.write(f"{dt} {axis} {n} {m} {ch} {spc}\n")


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--out", default="tuning_b200.txt")
    ap.add_argument("--dtypes", default="f64,f32")
    ap.add_argument("--lengths", default="32,64,128,256,512,1024,4096,65536")
    ap.add_argument("--elems", type=int, default=1 << 24)
    ap.add_argument("--classes", default="0,1,2,4",
                    help="axis classes to sweep (0-3 strided-batch strides, 4 variable-length)")
    ap.add_argument("--report", default=None, help="also write every timing as JSON")
    ap.add_argument("--stride-sweep", action="store_true",
                    help="only time strided solves against the plane stride")
    args = ap.parse_args()
    if args.stride_sweep:
        stride_sweep()
        return
    table, report = tune(args.dtypes.split(","), [int(v) for v in args.lengths.split(",")],
                         args.elems, classes=[int(v) for v in args.classes.split(",")])
    write_table(table, args.out)
    if args.report:
        with open(args.report, "w") as f:
            json.dump(report, f, indent=1)
    print(open(args.out).read())


if __name__ == "__main__":
    main()
