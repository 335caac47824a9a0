"""A small case of the hot path for ``ncu`` captures (a few GB on the device).

    python -m octrees_benchmark_b200.profile_case [--points N] [--queries Q]

Builds one synthetic tile (default 6M points at the 10M-point tile's density,
Hilbert keys, leaf 64), then answers Q radius queries (sphere, neighborsPrune,
r = 2.5 m) and Q kNN queries (k = 50) at random cloud points on the packet path,
twice (the second round is the one to capture).  Inputs exceed L2 (the cloud's
coordinates alone are 144 MB).  Prints one line with the result sizes.
"""
from __future__ import annotations

import argparse
import ctypes as C
import math


def main():
    import torch

    from . import capi
    from .linear_octree import LinearOctree
    from .synth import lidar_tile

    ap = argparse.ArgumentParser()
    ap.add_argument("--points", type=int, default=6_000_000)
    ap.add_argument("--queries", type=int, default=200_000)
    ap.add_argument("--fp32", action="store_true", help="FP32 leaf-relative filter on the radius search")
    args = ap.parse_args()
    n, q = args.points, args.queries
    xyz = lidar_tile(n, 1500.0 * math.sqrt(n / 10_000_000), 1)
    d = torch.from_numpy(xyz).cuda()
    oc = LinearOctree(d, encoder="hilbert", max_points_leaf=64, fp32_filter=args.fp32)
    _, _, s = oc.sorted_points()
    sd = torch.from_numpy(s).cuda()
    g = torch.Generator(device="cuda").manual_seed(5)
    qr = sd[torch.randint(0, n, (q,), device="cuda", generator=g)].contiguous()
    qk = sd[torch.randint(0, n, (q,), device="cuda", generator=g)].contiguous()
    torch.cuda.synchronize()
    L = capi.lib()
    MD = capi.OCT_MEM_DEVICE
    h = oc.handle
    offs = torch.zeros(q + 1, dtype=torch.int64, device="cuda")
    tot = C.c_uint64()
    L.oct_radius_search(h, 1, 2, qr.data_ptr(), q, None, 2.5, offs.data_ptr(), None, 0, C.byref(tot), MD)
    cap = int(tot.value) + 1024
    out = torch.empty(cap, dtype=torch.int32, device="cuda")
    kidx = torch.empty(q * 50, dtype=torch.int32, device="cuda")
    kd2 = torch.empty(q * 50, dtype=torch.float64, device="cuda")
    kc = torch.empty(q, dtype=torch.int32, device="cuda")
    for _ in range(2):
        capi.check(L.oct_radius_search(h, 1, 2, qr.data_ptr(), q, None, 2.5, offs.data_ptr(), out.data_ptr(), cap,
                                       C.byref(tot), MD), h)
        capi.check(L.oct_knn(h, qk.data_ptr(), q, 50, kidx.data_ptr(), kd2.data_ptr(), kc.data_ptr(), MD), h)
        capi.check(L.oct_synchronize(h), h)
    print(f"points {n} queries {q} radius results {tot.value} nodes {oc.n_total}")


if __name__ == "__main__":
    main()
