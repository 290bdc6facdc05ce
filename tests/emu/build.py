"""Builds the warp-emulation library of the decode engine's device logic (host g++ build, no GPU)."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(ROOT, "_build", "emu", "libfls_emu.so")
SRCS = [os.path.join(HERE, "emu_decode.cpp"), os.path.join(ROOT, "fastlanes_b200", "csrc", "fls_h_page.cpp")]
DEPS = SRCS + [os.path.join(ROOT, "fastlanes_b200", "csrc", f) for f in os.listdir(os.path.join(ROOT, "fastlanes_b200", "csrc"))
               if f.endswith((".h", ".cuh", ".cu", ".cpp"))] + [os.path.join(HERE, "include", "cuda_runtime.h")]


def build():
    if os.path.exists(OUT) and os.path.getmtime(OUT) >= max(os.path.getmtime(d) for d in DEPS):
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    cmd = ["g++", "-std=c++20", "-O1", "-shared", "-fPIC", "-pthread", "-DFLS_HOST_EMULATION=1", "-x", "c++",
           "-I" + os.path.join(HERE, "include"), "-I" + os.path.join(ROOT, "fastlanes_b200", "csrc"),
           "-I" + os.path.join(ROOT, "include"), "-o", OUT] + SRCS
    subprocess.check_call(cmd)
    return OUT
