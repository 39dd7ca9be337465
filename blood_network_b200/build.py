"""Build step: compiles the CUDA library in-tree for sm_100a.

``make -C blood_network_b200/csrc`` produces ``blood_network_b200/lib/
libamg_b200.so`` (nvcc -gencode arch=compute_100a,code=sm_100a -lineinfo).
"""
import os
import subprocess

_HERE = os.path.dirname(os.path.abspath(__file__))


def build(jobs: int = 8, verbose: bool = False) -> str:
    csrc = os.path.join(_HERE, "csrc")
    r = subprocess.run(["make", "-C", csrc, f"-j{jobs}"], capture_output=not verbose, text=True)
    if r.returncode != 0:
        raise RuntimeError("CUDA library build failed:\n" + (r.stdout or "") + (r.stderr or ""))
    return os.path.join(_HERE, "lib", "libamg_b200.so")


if __name__ == "__main__":
    print(build(verbose=True))
