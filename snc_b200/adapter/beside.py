"""Writes the reference's backend table with the B200 backends BESIDE its own.

    python beside.py <reference tree> <output dir>

The reference selects a forward backend by name through one enum and three
functions (include/snc/runtime.hpp:21-31, src/runtime/cpu_backend.cpp:14-37)
and dispatches in snc::forward (cpu_backend.cpp:195-207).  Extending that
table is the change a maintainer makes to add a backend, so this script
applies exactly that change to COPIES of three reference files, written
under <output dir> (a build folder, never committed):

  include/snc/runtime.hpp      Backend gains B200Atomic / B200Bucket /
                               B200Sort (values 5-7) and the hook namespace
                               snc::b200 (available, forward) beside
                               snc::cuda;
  src/runtime/cpu_backend.cpp  parse_backend / backend_name / backend_is_cuda
                               know "b200-atomic" / "b200-bucket" /
                               "b200-sort"; snc::forward sends those to
                               snc::b200::forward with the same CPU fallback
                               as the cuda-* backends;
  src/bench/snc_bench.cpp      --compare-backends also runs the b200-* rows.

Everything else -- the reference's CUDA backend (cuda_backend.cu), its
trainer, encoders, graph code -- is compiled unchanged from where it lies, so
one snc_bench run shows cpu, openmp, the reference's cuda-* kernels and the
b200-* rows side by side.  Each edit anchors on the text it extends and the
script fails if an anchor is missing, rather than guessing.
"""
from __future__ import annotations

import os
import sys

B200_NAMES = (("b200-atomic", "B200Atomic", 5), ("b200-bucket", "B200Bucket", 6),
              ("b200-sort", "B200Sort", 7))


def _insert_after(text: str, anchor: str, addition: str, path: str) -> str:
    if text.count(anchor) != 1:
        raise SystemExit(f"{path}: anchor not found exactly once: {anchor!r}")
    i = text.index(anchor) + len(anchor)
    return text[:i] + addition + text[i:]


def _replace(text: str, old: str, new: str, path: str) -> str:
    if text.count(old) != 1:
        raise SystemExit(f"{path}: text not found exactly once: {old!r}")
    return text.replace(old, new)


def runtime_hpp(text: str, path: str) -> str:
    enum = "".join(f"  {e} = {v},\n" for _, e, v in B200_NAMES)
    text = _insert_after(text, "  CudaSort = 4,\n", enum, path)
    hook = (
        "\n// ---- B200 backend hook (snc_b200 adapter), beside the CUDA backend ----\n"
        "namespace b200 {\n"
        "bool available();\n"
        "bool forward(const SNNGraph& g, const std::vector<InputEvent>& events,\n"
        "             int num_steps, const LIFParams& lif, Backend variant,\n"
        "             ForwardResult& out);\n"
        "}  // namespace b200\n")
    return _insert_after(text, "}  // namespace cuda\n", hook, path)


def cpu_backend_cpp(text: str, path: str) -> str:
    parse = "".join(f'  if (name == "{n}") {{ out = Backend::{e}; return true; }}\n'
                    for n, e, _ in B200_NAMES)
    text = _insert_after(text, '  if (name == "cuda-sort") { out = Backend::CudaSort; return true; }\n',
                         parse, path)
    names = "".join(f'    case Backend::{e}: return "{n}";\n' for n, e, _ in B200_NAMES)
    text = _insert_after(text, '    case Backend::CudaSort: return "cuda-sort";\n', names, path)
    text = _replace(text, "         b == Backend::CudaSort;\n",
                    "         b == Backend::CudaSort || b == Backend::B200Atomic ||\n"
                    "         b == Backend::B200Bucket || b == Backend::B200Sort;\n", path)
    dispatch = (
        "  if (backend == Backend::B200Atomic || backend == Backend::B200Bucket ||\n"
        "      backend == Backend::B200Sort) {\n"
        "    ForwardResult out;\n"
        "    if (b200::available() && b200::forward(g, events, num_steps, lif, backend, out))\n"
        "      return out;\n"
        "    return run_cpu(g, events, num_steps, lif, /*use_omp=*/false);\n"
        "  }\n")
    return _insert_after(text, "int num_steps, const LIFParams& lif, Backend backend) {\n", dispatch, path)


def snc_bench_cpp(text: str, path: str) -> str:
    return _replace(text, '{"cpu", "openmp", "cuda-atomic", "cuda-bucket", "cuda-sort"}',
                    '{"cpu", "openmp", "cuda-atomic", "cuda-bucket", "cuda-sort", '
                    '"b200-atomic", "b200-bucket", "b200-sort"}', path)


EDITS = {
    os.path.join("include", "snc", "runtime.hpp"): runtime_hpp,
    os.path.join("src", "runtime", "cpu_backend.cpp"): cpu_backend_cpp,
    os.path.join("src", "bench", "snc_bench.cpp"): snc_bench_cpp,
}


def main(ref: str, out: str) -> int:
    for rel, edit in EDITS.items():
        src = os.path.join(ref, rel)
        with open(src) as f:
            text = f.read()
        dst = os.path.join(out, rel)
        os.makedirs(os.path.dirname(dst), exist_ok=True)
        new = edit(text, src)
        old = open(dst).read() if os.path.exists(dst) else None
        if new != old:  # keep the timestamp when nothing changed (make)
            with open(dst, "w") as f:
                f.write(new)
    return 0


if __name__ == "__main__":
    if len(sys.argv) != 3:
        raise SystemExit(__doc__)
    sys.exit(main(sys.argv[1], sys.argv[2]))
