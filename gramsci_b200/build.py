"""Build the in-tree native artefacts: libgramsci_cuda.so (nvcc, sm_100a) and
the `gramsci` command-line host.  nvcc cross-compiles without a GPU."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")


def build(jobs=8, verbose=False):
    cmd = ["make", "-C", CSRC, f"-j{jobs}"]
    if not verbose:
        cmd.insert(1, "-s")
    subprocess.check_call(cmd)


if __name__ == "__main__":
    build(verbose=True)
