"""Build the C++/OpenMP restatement of the force evaluation (test infrastructure).

``python -m oracle.build_cpu`` compiles ``oracle/cpu/force_cpu.cpp`` with g++
into ``oracle/liboracle_cpu.so``.  The library is a checker and the timed CPU
baseline; the product never loads it.  It targets x86-64-v3 (AVX2 + FMA), which
every host this runs on supports, so the same file serves this container and
the GPU hosts.
"""
from __future__ import annotations

import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "cpu" / "force_cpu.cpp"
OUT = HERE / "liboracle_cpu.so"
INCLUDE = HERE.parent / "include"


def build() -> Path:
    deps = [SRC, INCLUDE / "invdft_force.h"]
    if OUT.exists() and OUT.stat().st_mtime >= max(d.stat().st_mtime for d in deps):
        return OUT
    cmd = ["g++", "-O3", "-march=x86-64-v3", "-fopenmp", "-std=c++17", "-shared", "-fPIC",
           "-I", str(INCLUDE), str(SRC), "-o", str(OUT)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"g++ failed for {SRC.name}:\n{r.stdout}\n{r.stderr}")
    return OUT


if __name__ == "__main__":
    print(build())
