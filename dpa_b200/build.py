"""Build recipe of the native parts: the sm_100a CUDA library and the C++ host
pipeline.

    python -m dpa_b200.build            # builds everything in-tree

Outputs (git-ignored, shipped with the tree):
    dpa_b200/libdpa_b200.so     C ABI of include/dpa_b200.h (CUDA, sm_100a)
    dpa_b200/libdpa_host.so     host pipeline, HDF5/XDMF, JSON (dpa_b200/host/dpa_host.h)
    dpa_b200/bin/dpa_pipeline   drop-in for the reference's `dpa config.json`
"""
from __future__ import annotations

import hashlib
import os
import shutil
import subprocess
import sys
from pathlib import Path

PACKAGE = Path(__file__).resolve().parent
ROOT = PACKAGE.parent
CSRC = PACKAGE / "csrc"
HOST = PACKAGE / "host"
INCLUDE = ROOT / "include"
LIBRARY = PACKAGE / "libdpa_b200.so"
PIPELINE = PACKAGE / "bin" / "dpa_pipeline"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_SOURCES = ["capi.cu", "advect.cu", "advect_f32.cu", "advect_f32e.cu", "advect_f16.cu",
                "advect_bf16.cu", "emit.cu", "ftle.cu", "noalloc.cu", "serve.cu"]


def nvcc() -> str:
    for candidate in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if candidate and Path(candidate).exists():
            return candidate
    raise RuntimeError("nvcc not found")


def _digest(sources: list[Path], command: list[str]) -> str:
    """Hash of the sources' contents and of the build command."""
    h = hashlib.sha256()
    for s in sorted(sources):
        h.update(str(s.relative_to(ROOT)).encode())
        h.update(s.read_bytes())
    # The tree may sit elsewhere on another machine: paths inside it count
    # relative to its root.
    h.update(" ".join(command).replace(str(ROOT), "<root>").encode())
    return h.hexdigest()


def _stale(target: Path, sources: list[Path], command: list[str]) -> bool:
    """A target is rebuilt unless its stamp records the current sources and
    command (content, not timestamps: a tree copied with newer modification
    times than its sources still rebuilds when the sources changed)."""
    stamp = target.with_name(target.name + ".stamp")
    if not target.exists() or not stamp.exists():
        return True
    return stamp.read_text().strip() != _digest(sources, command)


def _stamp(target: Path, sources: list[Path], command: list[str]) -> None:
    target.with_name(target.name + ".stamp").write_text(_digest(sources, command) + "\n")


def _run(cmd: list[str]) -> None:
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build_library(force: bool = False, verbose_ptxas: bool = False,
                  defines: tuple[str, ...] = ()) -> Path:
    sources = [CSRC / s for s in CUDA_SOURCES]
    deps = sources + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.hpp")) + \
        [INCLUDE / "dpa_b200.h"]
    flags = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
                    "-I", str(INCLUDE), "-I", str(CSRC), "--expt-relaxed-constexpr"]
    flags += [f"-D{d}" for d in defines]
    if not force and not _stale(LIBRARY, deps, flags):
        return LIBRARY
    build_dir = PACKAGE / "_build"
    build_dir.mkdir(exist_ok=True)
    objects = []
    compile_flags = flags + (["-Xptxas", "-v"] if verbose_ptxas else [])
    # The translation units compile in parallel (the advection kernel's
    # instantiations dominate and are split by field storage).
    from concurrent.futures import ThreadPoolExecutor
    commands = []
    for src in sources:
        obj = build_dir / (src.stem + ".o")
        commands.append([nvcc(), "-c", str(src), "-o", str(obj)] + compile_flags)
        objects.append(str(obj))
    with ThreadPoolExecutor(max_workers=min(len(commands), os.cpu_count() or 1)) as pool:
        for f in [pool.submit(_run, c) for c in commands]:
            f.result()
    tmp = LIBRARY.with_suffix(".so.tmp")
    _run([nvcc()] + ARCH + ["-shared", "-o", str(tmp)] + objects + ["-cudart", "static"])
    os.replace(tmp, LIBRARY)
    _stamp(LIBRARY, deps, flags)
    return LIBRARY


HOST_LIBRARY = PACKAGE / "libdpa_host.so"
HOST_SOURCES = ["hdf5.cpp", "json.cpp", "pipeline.cpp", "host_api.cpp"]


def host_compiler() -> str:
    # The system g++ (the CXX of this image's environment may point at a
    # toolchain without its support files).
    return "/usr/bin/g++" if Path("/usr/bin/g++").exists() else (shutil.which("g++") or "g++")


def build_host(force: bool = False) -> Path:
    """libdpa_host.so (HDF5 / JSON / seeding / pipeline, C++17) and the
    dpa_pipeline executable, both linked against libdpa_b200.so."""
    sources = [HOST / s for s in HOST_SOURCES]
    deps = sources + sorted(HOST.glob("*.hpp")) + sorted(HOST.glob("*.h")) + [
        INCLUDE / "dpa_b200.h", LIBRARY]
    command = [host_compiler(), "-std=c++17", "-O2", "-Wall", "-fPIC", "-shared",
               "-I", str(INCLUDE), "-I", str(HOST)] + [str(s) for s in sources]
    if force or _stale(HOST_LIBRARY, deps, command):
        tmp = HOST_LIBRARY.with_suffix(".so.tmp")
        _run(command + ["-o", str(tmp), "-L", str(PACKAGE), "-ldpa_b200", "-Wl,-rpath,$ORIGIN"])
        os.replace(tmp, HOST_LIBRARY)
        _stamp(HOST_LIBRARY, deps, command)
    main = HOST / "main.cpp"
    main_deps = [main, HOST_LIBRARY, HOST / "pipeline.hpp"]
    main_command = [host_compiler(), "-std=c++17", "-O2", "-Wall", "-I", str(INCLUDE), "-I",
                    str(HOST), str(main)]
    if force or _stale(PIPELINE, main_deps, main_command):
        PIPELINE.parent.mkdir(exist_ok=True)
        _run(main_command + ["-o", str(PIPELINE), "-L", str(PACKAGE), "-ldpa_host", "-ldpa_b200",
                             "-Wl,-rpath,$ORIGIN/.."])
        _stamp(PIPELINE, main_deps, main_command)
    return HOST_LIBRARY


def build(force: bool = False) -> None:
    build_library(force=force)
    build_host(force=force)


if __name__ == "__main__":
    build(force="--force" in sys.argv)
