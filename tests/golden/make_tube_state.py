"""Writes the twisted-tube state the headline benchmark and the tube parity tests start from.

The 300 x 296 tube (88,800 vertices; end rings rotating at -/+2 rad/s, dt 1/100) is stepped from rest
by the CPU restatement of the Newton loop (oracle/newton_cpu.py: time_step, the reference's PCG stop
rule -- r.z < 1e-10 checked every 25 iterations, at most 100), so no GPU is involved in making it.
The positions and velocities after FRAME steps are stored as float32 (V, 3) arrays with the frame
number in tests/golden/tube88k_state.npz.

    python tests/golden/make_tube_state.py [--frame 56] [--keep-dir DIR]

--keep-dir also writes every intermediate frame there (for choosing the frame).
"""
from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

OUT = os.path.join(HERE, "tube88k_state.npz")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--frame", type=int, default=56)
    ap.add_argument("--keep-dir", default=None)
    a = ap.parse_args()
    from luisacomputesimulator_b200 import scenes as S
    from oracle import newton_cpu as N
    from oracle import oracle as O

    sc = S.twisted_tube(300, 296)
    pat = N.MaterialPattern(sc)
    x = sc.x.copy()
    v = np.zeros_like(x)
    for f in range(a.frame):
        t0 = time.perf_counter()
        x, v, recs = N.time_step(sc, x, v, f, pattern=pat)
        print(f"frame {f + 1}: {time.perf_counter() - t0:.1f} s, "
              + ", ".join(f"(pcg {r['pcg_iters']}, toi {r['toi']:.4f}, vf {r['vf']}, ee {r['ee']}, pairs {r['pairs']})"
                          for r in recs), flush=True)
        if a.keep_dir:
            os.makedirs(a.keep_dir, exist_ok=True)
            np.savez(os.path.join(a.keep_dir, f"frame{f + 1}.npz"), x=x[:, :3], v=v[:, :3], frame=f + 1)
    d = O.min_distance(sc, x)
    print(f"min distance at frame {a.frame}: {d:.3e}")
    assert d > 0.0
    np.savez_compressed(OUT, x=np.ascontiguousarray(x[:, :3], np.float32),
                        v=np.ascontiguousarray(v[:, :3], np.float32), frame=np.int32(a.frame))
    print(OUT)


if __name__ == "__main__":
    main()
