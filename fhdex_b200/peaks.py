"""Measured FMA throughput (FP64 and FP32) of a GPU, through ``fhd_measure_fma_peak``.

The HBM denominator of the step's roofline is the driver-measured copy bandwidth
(``MEASURED_PEAKS.json``); the compute denominator is measured here, with the
same rules: CUDA-event timing, no change of clocks or power settings.
``python -m fhdex_b200.peaks [device] [path]`` writes the figures and the SM
clock seen after measuring as JSON (default path: ``MEASURED_FMA.json`` at the
repository root).
"""
from __future__ import annotations

import ctypes as C
import json
import os
import subprocess
import sys

from . import capi


def measure_fma_peaks(device: int = 0) -> dict:
    lib = capi.load()
    out = {}
    for name, fp64 in (("fp64_tflops", 1), ("fp32_tflops", 0)):
        v = C.c_double()
        capi.check(lib.fhd_measure_fma_peak(device, fp64, C.byref(v)), "fhd_measure_fma_peak")
        out[name] = v.value
    return out


def _clock(device: int):
    try:
        r = subprocess.run(["nvidia-smi", "-i", str(device), "--query-gpu=clocks.sm,clocks.max.sm,name",
                            "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=20)
        sm, smax, name = [x.strip() for x in r.stdout.strip().split(",")]
        return {"sm_mhz_after": float(sm), "sm_max_mhz": float(smax), "gpu": name}
    except Exception:
        return {}


def main(argv):
    import torch
    dev = int(argv[1]) if len(argv) > 1 else 0
    torch.cuda.init()
    best = {"fp64_tflops": 0.0, "fp32_tflops": 0.0}
    for _ in range(3):
        m = measure_fma_peaks(dev)
        best = {k: max(best[k], m[k]) for k in best}
    best.update(_clock(dev))
    best["method"] = ("best of 3x5 CUDA-event-timed launches of 8 independent fma chains per thread, "
                      "whole waves of 256-thread blocks (fhd_measure_fma_peak); 2 flops per fma")
    path = argv[2] if len(argv) > 2 else os.path.join(
        os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "MEASURED_FMA.json")
    with open(path, "w") as f:
        json.dump(best, f, indent=1)
    print(json.dumps(best))


if __name__ == "__main__":
    main(sys.argv)
