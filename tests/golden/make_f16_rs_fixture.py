"""Builds tests/golden/f16_rs_probe.npz: the GPU's cvt.rs.f16x2.f32 outputs
for seeded inputs, the pin of the FP16S stochastic rounding restated in the
oracle (orc_f16_rs).  Needs nvcc and a B200.

Usage: python tests/golden/make_f16_rs_fixture.py [--out-dir DIR]
"""
import argparse
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out-dir", default=HERE)
    a = ap.parse_args()
    with tempfile.TemporaryDirectory() as d:
        exe = os.path.join(d, "probe")
        subprocess.run(["nvcc", "-O2", "-gencode", "arch=compute_100a,code=sm_100a",
                        os.path.join(HERE, "f16_rs_probe.cu"), "-o", exe], check=True)
        binf = os.path.join(d, "probe.bin")
        subprocess.run([exe, binf], check=True)
        raw = np.fromfile(binf, dtype=np.uint32)
    n = raw.size // 4
    va, vb, r, o = raw[:n], raw[n:2 * n], raw[2 * n:3 * n], raw[3 * n:]
    sel = np.concatenate([np.nonzero(np.arange(n) % 4 == g)[0][:2048] for g in range(4)])
    np.savez_compressed(os.path.join(a.out_dir, "f16_rs_probe.npz"), a=va[sel], b=vb[sel], r=r[sel], out=o[sel])


if __name__ == "__main__":
    main()
