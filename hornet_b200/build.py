"""Build the in-tree sm_100a library (hornet_b200/_lib/libhornet_b200.so).

    python -m hornet_b200.build

nvcc cross-compiles for sm_100a without a GPU.  Objects go to
hornet_b200/csrc/_build/ (git-ignored)."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def build(jobs: int = 8) -> str:
    subprocess.run(["make", "-C", os.path.join(HERE, "csrc"), f"-j{jobs}"], check=True)
    return os.path.join(HERE, "_lib", "libhornet_b200.so")


if __name__ == "__main__":
    print(build(int(sys.argv[1]) if len(sys.argv) > 1 else 8))
