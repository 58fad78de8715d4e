"""FP64 tensor-core probe of this GPU: mma latency, issue interval and throughput.

    python -m gbskernels_b200.probe

One JSON line per shape: k (m16n8k8 or m16n8k4), independent accumulator chains
per warp, warps per SM (one block per SM on every SM), TFLOP/s and warp 0's cycles
per mma (for one chain on one warp: the mma's latency).  The roofline denominator
of the hafnian kernel is the saturated rate; the latency and issue interval tell
how many chains a warp needs to keep the pipe full.
"""

from __future__ import annotations

import json

import numpy as np

from . import _lib

SHAPES = [  # (k, chains, warps per SM, blocks: 0 = one per SM)
    (8, 1, 1, 1), (4, 1, 1, 1),
    (8, 1, 4, 0), (8, 2, 4, 0), (8, 4, 4, 0), (8, 8, 4, 0), (4, 4, 4, 0),
    (8, 1, 8, 0), (8, 2, 8, 0), (8, 4, 8, 0), (8, 1, 12, 0), (8, 1, 16, 0),
]


def sweep(shapes=SHAPES) -> list[dict]:
    import torch
    lib = _lib.load()
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    out = []
    for k, ch, w, blocks in shapes:
        tf = np.zeros(1)
        cyc = np.zeros(1)
        _lib.check(lib.gbs_probe_fp64_mma_chains(k, ch, w, blocks or sms, _lib.dptr(tf), _lib.dptr(cyc)),
                   "gbs_probe_fp64_mma_chains")
        out.append({"k": k, "chains_per_warp": ch, "warps_per_sm": w, "blocks": blocks or sms,
                    "tflops": float(tf[0]), "cycles_per_mma": float(cyc[0])})
    return out


if __name__ == "__main__":
    for row in sweep():
        print(json.dumps(row), flush=True)
