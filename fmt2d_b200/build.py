"""Build the native libraries for sm_100a (nvcc cross-compiles without a GPU):
the C-ABI library (fmt2d_b200/_lib/libfmt2d_b200.so) and the PyTorch
operators on it (fmt2d_b200/_lib/libfmt2d_torch.so, torch.ops.fmt2d.*)."""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_lib")
TORCH_OPS = os.path.join(LIB, "libfmt2d_torch.so")


def build(jobs: int = 8) -> str:
    subprocess.run(["make", "-s", "-j", str(jobs), "-C", os.path.join(HERE, "csrc")], check=True)
    build_torch_ops()
    return os.path.join(LIB, "libfmt2d_b200.so")


def build_torch_ops() -> str:
    """Compile csrc/torch_ops.cpp against torch and libfmt2d_b200.so (in-tree,
    rpath to _lib) into _lib/libfmt2d_torch.so.  The compile runs in a child
    process: torch.utils.cpp_extension loads what it builds, and a second
    library registering the fmt2d operators in the caller's process would
    abort it."""
    src = os.path.join(HERE, "csrc", "torch_ops.cpp")
    if os.path.exists(TORCH_OPS) and os.path.getmtime(TORCH_OPS) >= max(
            os.path.getmtime(src), os.path.getmtime(os.path.join(LIB, "libfmt2d_b200.so"))):
        return TORCH_OPS
    bdir = os.path.join(HERE, "_build", "torch_ops")
    os.makedirs(bdir, exist_ok=True)
    # The link line runs under ninja and a shell: $$ is ninja's literal dollar
    # sign, the quotes keep the shell from expanding $ORIGIN.
    code = (
        "import sys\n"
        "from torch.utils import cpp_extension as ce\n"
        "out = ce.load(name='fmt2d_torch', sources=[sys.argv[1]], build_directory=sys.argv[2],\n"
        "              is_python_module=False, with_cuda=True, verbose=False,\n"
        "              extra_cflags=['-O2', '-std=c++17'],\n"
        "              extra_ldflags=['-L' + sys.argv[3], '-lfmt2d_b200',\n"
        "                             \"'-Wl,-rpath,$$ORIGIN'\", \"'-Wl,-rpath,$$ORIGIN/../../_lib'\"])\n")
    subprocess.run([sys.executable, "-c", code, src, bdir, LIB], check=True)
    shutil.copy2(os.path.join(bdir, "fmt2d_torch.so"), TORCH_OPS)
    return TORCH_OPS


if __name__ == "__main__":
    print(build())
