"""Build recipe of the CPU oracle (test infrastructure; see prism_oracle.cpp).

Compiles oracle/prism_oracle.cpp with g++ -O2 (the reference's CMake release
flag, CMakeLists.txt:30-37; no -march, so no FMA contraction) into
oracle/liboracle.so.
"""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "prism_oracle.cpp")
HDR = os.path.join(HERE, "..", "include", "prism_b200.h")
LIB = os.path.join(HERE, "liboracle.so")


def build(force=False):
    newest = max(os.path.getmtime(SRC), os.path.getmtime(HDR))
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= newest:
        return LIB
    cmd = ["g++", "-std=c++20", "-O2", "-fPIC", "-shared", "-fvisibility=hidden",
           "-ffp-contract=off", "-o", LIB + ".tmp", SRC]
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force=True))
