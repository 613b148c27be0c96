"""Makes the reference CUDA benchmark's hierarchize7 kernel safe to run, for
timing next to this project's kernels.  TEST INFRASTRUCTURE ONLY: run by
oracle/Makefile, it reads adaptive_sparse_grid_bench_cuda.cu where it lies
and writes a patched copy into oracle/_ref/ (git-ignored, never committed).

hierarchize7 (adaptive_sparse_grid_bench_cuda.cu:1053-1160) runs one warp
per chain of subspaces along the current dimension.  Lane 0 writes the
chain's level vector, parent offsets and prefix sums to shared memory and
decrements the current level at the end of each step; the other lanes read
them with no barrier between (the source relies on warp-synchronous
execution, which independent thread scheduling does not give).  The patch
adds a __syncwarp() at each of those hand-overs and changes nothing else:
  1. before the loop over the chain's levels (after lane 0 set up the
     levels and parent offsets, cu:1080-1097);
  2. after lane 0 wrote the prefix sums of a step (cu:1103-1108);
  3. around lane 0's decrement of the level at the end of a step
     (cu:1155-1156): every lane has finished the step's updates before the
     level changes, and sees the new level before the next step.
With these, the updates of a step and the parent reads of the next are
ordered too (__syncwarp orders memory among the lanes it joins).  The
barriers need all 32 lanes: every warp of a launch is whole when a
finest-level subspace holds >= 32 points (n >= 6), and the harness refuses
smaller n.

Each replacement must match exactly once inside hierarchize7, or the script
fails and no patched file is written.

usage: patch_ref_cuda.py REF_CU OUT
"""
import re
import sys


def patch(src: str) -> str:
    start = src.index("__global__ void hierarchize7(")
    end = src.index("__global__", start + 1)
    body = src[start:end]
    rules = [
        (r"for \(; levels\[crt_dim\] >= 1;", r"__syncwarp(); for (; levels[crt_dim] >= 1;"),
        (r"(prefix_sums\[l\] = prefix_sums\[l \+ 1\] \+ levels\[l\];\s*\n\s*\})", r"\1 __syncwarp();"),
        (r"if \(0 == lane\)\s*\n\s*--levels\[crt_dim\];",
         r"__syncwarp(); if (0 == lane) --levels[crt_dim]; __syncwarp();"),
    ]
    for pat, rep in rules:
        body, k = re.subn(pat, rep, body)
        if k != 1:
            raise SystemExit(f"patch_ref_cuda: pattern {pat!r} matched {k} times in hierarchize7")
    return src[:start] + body + src[end:]


def main() -> None:
    ref_cu, out = sys.argv[1], sys.argv[2]
    with open(ref_cu) as f:
        src = f.read()
    patched = patch(src)
    with open(out, "w") as f:
        f.write(patched)


if __name__ == "__main__":
    main()
