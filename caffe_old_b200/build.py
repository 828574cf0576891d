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


def reference_root() -> str:
    """Where the reference's sources are looked for: the oracle recipe's REF (environment variable
    CAFFE_REFERENCE, else the recipe's default)."""
    r = subprocess.run(["make", "-C", os.path.join(_ROOT, "oracle"), "-s", "--no-print-directory", "refpath"],
                       capture_output=True, text=True, check=True)
    return r.stdout.strip()


def build_oracle_ref(reference: str | None = None) -> bool:
    """The reference's own geometry sources and its solver path (with stand-in PETSc / MPI /
    LAPACKE / Boost headers), compiled where they lie into oracle/_ref/: pins for the oracle.
    Returns False when the reference sources are not present."""
    reference = reference or reference_root()
    if not os.path.exists(os.path.join(reference, "src", "Math", "Geometry.cpp")):
        return False
    subprocess.run(["make", "-C", os.path.join(_ROOT, "oracle"), "-s", "-j8", "ref", "refsolver", f"REF={reference}"], check=True)
    return True


def build_all() -> None:
    build_device()
    build_host()
    build_oracle()
    build_oracle_ref()


if __name__ == "__main__":
    build_all()
