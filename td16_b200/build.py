"""Builds libtd16b200.so in-tree with nvcc for sm_100a (and the JNI shim when a
JDK's jni.h is available).  Usage: python -m td16_b200.build [--verbose]"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libtd16b200.so")
JNI_LIB = os.path.join(PKG, "libtd16_jni.so")
THREADS_LIB = os.path.join(PKG, "libtd16_slot_threads.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-fvisibility=hidden",
              "-shared", "--expt-relaxed-constexpr"]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build td16_b200")
    return cand


def _sources():
    return [os.path.join(CSRC, "td_engine.cu"), os.path.join(CSRC, "td_cert.cu"), os.path.join(CSRC, "td_batcher.cc")]


def _deps():
    return [p for p in glob.glob(os.path.join(CSRC, "*")) if p.endswith((".cu", ".cuh", "td_batcher.cc"))] + [
        os.path.join(PKG, "..", "include", "td16_b200.h")]


def up_to_date(target: str, deps=None) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in (deps if deps is not None else _deps()) if os.path.exists(d))


def build(verbose: bool = False, force: bool = False) -> str:
    if force or not up_to_date(LIB):
        cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-I", CSRC, "-I", os.path.join(PKG, "..", "include"), "-o", LIB,
               *_sources(), "-lcudart"]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        res = subprocess.run(cmd, capture_output=True, text=True)
        if verbose or res.returncode != 0:
            sys.stderr.write(res.stdout + res.stderr)
        if res.returncode != 0:
            raise RuntimeError("nvcc failed building libtd16b200.so")
    _build_slot_threads(verbose, force)
    _build_jni(verbose)
    return LIB


def _build_slot_threads(verbose: bool, force: bool) -> None:
    """Native slot threads that drive a blocking search entry (td_slot_threads.cc)."""
    src = os.path.join(CSRC, "td_slot_threads.cc")
    if not force and up_to_date(THREADS_LIB, [src]):
        return
    cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-pthread", "-fvisibility=hidden", "-o", THREADS_LIB, src]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if verbose or res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
    if res.returncode != 0:
        raise RuntimeError("g++ failed building libtd16_slot_threads.so")


def _jni_include():
    home = os.environ.get("JAVA_HOME")
    roots = [home] if home else []
    roots += glob.glob("/usr/lib/jvm/*")
    for r in roots:
        inc = os.path.join(r, "include")
        if os.path.exists(os.path.join(inc, "jni.h")):
            return [inc, os.path.join(inc, "linux")]
    return None


def _build_jni(verbose: bool) -> None:
    """The JNI shim is only built where a JDK provides jni.h (as the reference's
    CMake builds td16_jni only if(JNI_FOUND))."""
    inc = _jni_include()
    if inc is None:
        return
    src = os.path.join(CSRC, "td_jni.cc")
    cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", *[f"-I{p}" for p in inc],
           "-I", os.path.join(PKG, "..", "include"), "-o", JNI_LIB, src,
           f"-L{PKG}", "-ltd16b200", "-Wl,-rpath,$ORIGIN"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if verbose or res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
    if res.returncode != 0:
        raise RuntimeError("g++ failed building libtd16_jni.so")


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, force="--force" in sys.argv)
    print(LIB)
