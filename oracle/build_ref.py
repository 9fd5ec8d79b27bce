"""Build the reference `svraster_cuda._C` extension from its own sources, in place,
into ``oracle/_ref/`` (test infrastructure only; never imported by the product).

The reference sources are read where they lie (``<reference>/cuda``); nothing is
copied into this repository.  The build recipe here is our own: it compiles the
same translation units the reference lists (cuda/setup.py:20-34) for sm_100a only.
The resulting ``svraster_ref_C*.so`` travels to the GPU machine with the rest of the
tree and is loaded there by ``oracle/ref_loader.py`` to produce golden fixtures and
the per-view reference timing.

Usage:  python oracle/build_ref.py [/path/to/reference]
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")

SOURCES = [
    "src/raster_state.cu", "src/preprocess.cu", "src/forward.cu", "src/backward.cu",
    "src/geo_params_gather.cu", "src/sh_compute.cu", "src/tv_compute.cu",
    "src/vg_compute.cu", "src/ge_compute.cu", "src/ls_compute.cu",
    "src/pl_compute.cu", "src/utils.cu", "src/adam_step.cu", "binding.cpp",
]


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SVR_REFERENCE_DIR")
    if not ref:
        print("no reference checkout given (argument or SVR_REFERENCE_DIR); nothing to build")
        return 0
    cuda_dir = os.path.join(ref, "cuda")
    if not os.path.isdir(cuda_dir):
        print(f"reference sources not found at {cuda_dir}; nothing to build")
        return 0
    os.makedirs(OUT, exist_ok=True)
    os.environ.setdefault("TORCH_CUDA_ARCH_LIST", "10.0a")
    os.environ.setdefault("MAX_JOBS", "4")
    from torch.utils.cpp_extension import load
    if not os.path.exists(os.path.join(OUT, "svraster_ref_C.so")):
        load(
            name="svraster_ref_C",
            sources=[os.path.join(cuda_dir, s) for s in SOURCES],
            build_directory=OUT,
            extra_cuda_cflags=["-O3"],
            extra_cflags=["-O3"],
            verbose=True,
        )
    # The smoothness adjoints once more, unmodified, with a compile prelude that fixes the
    # clock64() seed so their output can be pinned (oracle/ref_seeded/prelude.cuh).
    seeded = os.path.join(OUT, "seeded")
    os.makedirs(seeded, exist_ok=True)
    if not os.path.exists(os.path.join(seeded, "svraster_ref_seeded_C.so")):
        prelude = os.path.join(HERE, "ref_seeded", "prelude.cuh")
        load(
            name="svraster_ref_seeded_C",
            sources=[os.path.join(cuda_dir, "src/ls_compute.cu"), os.path.join(cuda_dir, "src/ge_compute.cu"),
                     os.path.join(HERE, "ref_seeded", "binding.cpp")],
            build_directory=seeded,
            extra_cuda_cflags=["-O3", "-include", prelude],
            extra_cflags=["-O3"],
            extra_include_paths=[os.path.join(cuda_dir, "src")],
            verbose=True,
        )
    print("built", OUT)
    return 0


if __name__ == "__main__":
    sys.exit(main())
