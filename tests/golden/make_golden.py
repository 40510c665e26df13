"""Write the golden fixtures: the oracle's results on small seeded synthetic
stacks (the library's host generator, so the inputs are rebuilt from a seed).

Run from the repository root after building both libraries:
    python tests/golden/make_golden.py
Each case stores the input's hash, the fused u16 image, the winner map, the
transforms, gains, shares, crop and (with the depth pass) the depth map and
the noise-floor cells, compressed. The CPU tests check that the oracle still
reproduces them; the GPU tests check the CUDA path against them.
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

CASES = {
    # name: (w, h, n, synth options, align?, depth?, fuse options)
    "plain_6x160x112": (160, 112, 6, dict(seed=101, mag_step=0.002), False, True, {}),
    "aligned_5x192x128": (192, 128, 5, dict(seed=202, warp=True, mag_step=0.0), True, True, {}),
    "chroma_4x128x96_nodepth": (128, 96, 4, dict(seed=303, mag_step=0.003), False, False, dict(use_chroma=True, levels=4)),
}


def inputs(case):
    import lapstack_b200 as L
    w, h, n, sy, _, _, _ = CASES[case]
    fr, _ = L.synth_stack(L.SynthSpec(w, h, n, **sy))
    return fr


def params(case, mod):
    _, _, _, _, align, depth, fuse = CASES[case]
    return (mod.FuseParams(**fuse), mod.AlignParams(coarsen=1) if align else None, mod.DepthParams() if depth else None)


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main():
    from oracle import oracle as O
    for case in CASES:
        fr = inputs(case)
        fp, ap, dp = params(case, O)
        r = O.run_stack(fr, O.StackParams(fuse=fp, align=ap, depth=dp))
        out = dict(input_sha256=np.array(digest(fr)), image_u16=r.image_u16, winner=r.winner, sims=r.sims, gains=r.gains,
                   shares=r.shares, crop=np.array(r.stats["crop"]), levels=np.array(r.stats["levels"]))
        if r.depth is not None:
            out.update(depth=r.depth.astype(np.float32), floor_cells=r.floor_cells.astype(np.float32))
        np.savez_compressed(os.path.join(HERE, f"{case}.npz"), **out)
        print(case, os.path.getsize(os.path.join(HERE, f"{case}.npz")), "bytes")


if __name__ == "__main__":
    main()
