"""The JNI shim (td16_b200/csrc/td_jni.cc) without a JVM: it is compiled
against a minimal hand-written jni.h (tests/jni/jni.h) and driven through a
fake JNIEnv (tests/jni/jni_driver.cc), the way GPUSortingSearch.java calls its
natives (jni_sorter.cu:24-117 is the reference shim).

  fake engine   every engine status mapped to its RuntimeException, int[][]
                shapes, argument pass-through, the batch native and the pair
                consumer natives (no GPU)
  real engine   linked to libtd16b200.so: argument checks and initialisation
                failure without a GPU; real searches with one, per call, in a
                batch and through the pair consumer with its certificate file
"""
import os
import subprocess

import pytest

from tests.conftest import has_gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = [os.path.join(ROOT, "td16_b200", "csrc", "td_jni.cc"), os.path.join(ROOT, "tests", "jni", "jni_driver.cc")]
INC = ["-I", os.path.join(ROOT, "tests", "jni"), "-I", os.path.join(ROOT, "include")]


def _build(tmp_path, fake: bool) -> str:
    out = str(tmp_path / ("jni_fake" if fake else "jni_real"))
    cmd = ["g++", "-O1", "-std=c++17", "-Wall", *INC, "-o", out, *SRC]
    if fake:
        cmd.insert(1, "-DTD_FAKE_ENGINE")
    else:
        lib = os.path.join(ROOT, "td16_b200")
        cmd += [f"-L{lib}", "-ltd16b200", f"-Wl,-rpath,{lib}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return out


def _run(binary, mode):
    p = subprocess.run([binary, mode], capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout + p.stderr
    assert "jni ok" in p.stdout, p.stdout
    return p.stdout


def test_shim_maps_every_status_without_a_jvm(tmp_path):
    out = _run(_build(tmp_path, fake=True), "fake")
    assert int(out.split("jni ok ")[1].split()[0]) >= 20


def test_shim_against_the_engine_without_a_gpu(tmp_path, td):
    if has_gpu():
        pytest.skip("this machine has a GPU: the real-engine case runs in the gpu test")
    _run(_build(tmp_path, fake=False), "real-cpu")


@pytest.mark.gpu
def test_shim_against_the_engine_on_the_gpu(tmp_path, td):
    out = _run(_build(tmp_path, fake=False), "real-gpu")
    assert int(out.split("jni ok ")[1].split()[0]) >= 200
