"""Recipe (measurement infrastructure, not the product): the reference's own
CUDA kernels, as its GPU path compiles them, for timing on this GPU.

crates/lapstack-core/src/gpu.rs holds its kernels as CUDA C source in three
string constants (COMMON, SRC, DEPTH_SRC) that it compiles at run time with
NVRTC for compute_86 (gpu.rs:312-318) into two modules: COMMON + SRC (the
fuser and the aligned frames) and COMMON + DEPTH_SRC (the depth pass). This
script reads those strings from the reference tree where they lie and writes
the two modules' sources, unchanged, under oracle/_ref/; `make ref` then
compiles each to PTX for compute_86 (which the driver JIT-compiles at load,
as it does NVRTC's PTX) and builds oracle/ref_gpu_harness.cpp, which loads
the modules through the driver API and drives them in the reference's host
order. Nothing is written into the repository's tracked tree, and
oracle/_ref/ is not committed.

Usage: python oracle/ref_gpu.py [path/to/gpu.rs] [outdir]
"""
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_SRC = "/root/reference/crates/lapstack-core/src/gpu.rs"


def strings(text):
    """The raw string constants of a Rust file: name -> contents (r#"..."#)."""
    out = {}
    for m in re.finditer(r'const ([A-Z_]+): &str = r#"', text):
        start = m.end()
        end = text.index('"#;', start)
        out[m.group(1)] = text[start:end]
    return out


def main(argv):
    src = argv[1] if len(argv) > 1 else DEFAULT_SRC
    outdir = argv[2] if len(argv) > 2 else os.path.join(HERE, "_ref")
    with open(src) as f:
        s = strings(f.read())
    missing = [k for k in ("COMMON", "SRC", "DEPTH_SRC") if k not in s]
    if missing:
        raise SystemExit(f"{src}: no {', '.join(missing)} string")
    os.makedirs(outdir, exist_ok=True)
    for name, body in (("ref_fuse.cu", s["COMMON"] + s["SRC"]), ("ref_depth.cu", s["COMMON"] + s["DEPTH_SRC"])):
        with open(os.path.join(outdir, name), "w") as f:
            f.write(f"// generated by oracle/ref_gpu.py from {src} (gpu.rs's NVRTC module source); not committed\n")
            f.write(body)
    print(outdir)


if __name__ == "__main__":
    main(sys.argv)
