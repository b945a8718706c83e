"""Compiles the C++ examples of tests/cpp against include/ and the built library."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "dioma-core_b200")


def build(name: str) -> str:
    src = os.path.join(ROOT, "tests", "cpp", name + ".cpp")
    out = os.path.join(ROOT, "tests", "cpp", name)
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), src,
                           "-L", LIBDIR, "-lsimuse_b200", "-Wl,-rpath," + LIBDIR, "-o", out])
    return out
