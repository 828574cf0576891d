"""In-tree build of the native parts: the sm_100a device library (csrc/), the C++ host
layer and module executables (host/), and the CPU oracle used by the tests (oracle/).  Both are plain Makefiles; nvcc cross-compiles
without a GPU."""
from __future__ import annotations

import os
import subprocess

_HERE = os.path.dirname(os.path.abspath(__file__))
_ROOT = os.path.dirname(_HERE)


def build_device(jobs: int = 8) -> str:
    subprocess.run(["make", "-C", os.path.join(_HERE, "csrc"), f"-j{jobs}", "-s"], check=True)
    return os.path.join(_HERE, "_build", "libcaffe_b200.so")


def build_host(jobs: int = 8) -> str:
    """The C++ host layer (solver / mesh / input interface over the device library) and the
    module executables caffeSimple, caffePiso, caffeIbPiso, hexaMesh, caffeCaseInfo."""
    subprocess.run(["make", "-C", os.path.join(_HERE, "host"), f"-j{jobs}", "-s"], check=True)
    return os.path.join(_HERE, "_build", "bin")


def build_oracle() -> str:
    subprocess.run(["make", "-C", os.path.join(_ROOT, "oracle"), "-s"], check=True)
    return os.path.join(_ROOT, "oracle", "_build", "liboracle.so")


def build_all() -> None:
    build_device()
    build_host()
    build_oracle()


if __name__ == "__main__":
    build_all()
