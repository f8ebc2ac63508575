"""CPU check of the ghost-frame copy's index mapping (no GPU needed).

Every upload copies the ghost frame of the state into the two stage buffers
(k_copy_frame), so that ghost cells no boundary operator writes keep their
uploaded values whichever buffer holds the state.  tests/emu/emu_frame.cu
compiles the mapping the kernel uses (frame_cells / frame_offset) for the
host and checks, for several shapes and pitches, that it covers every cell
within two of an edge in all four planes exactly once and nothing else."""
import os
import shutil
import subprocess
import tempfile

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
NVCC = "/usr/local/cuda/bin/nvcc"


def test_frame_mapping_covers_the_ghost_frame_once():
    if not os.path.exists(NVCC):
        pytest.skip("nvcc not available")
    d = tempfile.mkdtemp()
    try:
        exe = os.path.join(d, "emu_frame")
        subprocess.check_call([NVCC, "-std=c++17", "-O1", "-w",
                               "-gencode", "arch=compute_100a,code=sm_100a",
                               "-I", os.path.join(ROOT, "include"),
                               "-o", exe, os.path.join(HERE, "emu", "emu_frame.cu")])
        out = subprocess.run([exe], capture_output=True, text=True, timeout=120)
        print(out.stdout)
        assert out.returncode == 0, out.stdout + out.stderr
        assert out.stdout.strip().endswith("bad 0")
    finally:
        shutil.rmtree(d, ignore_errors=True)
