"""A compiled C program drives the device path through the C ABI alone
(tests/c/abi_device_calls.c: gcc, include/afhe.h, -lafhe): NTT round trip,
elementwise operators against the host, afhe_dispatch OP 99 then OP 3,
rotations and relinearisation against their batched forms."""
import os
import shutil
import subprocess

import pytest

from anns_fhe_b200 import build as B

pytestmark = pytest.mark.gpu


def test_c_program_drives_the_device_path():
    if shutil.which("gcc") is None:
        pytest.skip("gcc absent")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    libdir = os.path.join(root, "anns_fhe_b200", "lib")
    B.build()
    out_dir = os.path.join(root, "tests", "c", "_build")
    os.makedirs(out_dir, exist_ok=True)
    exe = os.path.join(out_dir, "abi_device_calls")
    subprocess.run(["gcc", "-std=c11", "-O1", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(root, "include"),
                    os.path.join(root, "tests", "c", "abi_device_calls.c"), "-L", libdir, "-lafhe",
                    f"-Wl,-rpath,{libdir}", "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    assert r.stdout.splitlines() == ["ntt round trip ok", "poly_add / poly_mul_ntt ok", "afhe_dispatch ok",
                                     "rotations ok", "mult_relin_rescale ok", "all ok"]
