"""The drop-in: the reference's unmodified CLI (src/main.c) linked with
-Wl,--wrap=pathtrace_render,--wrap=render_image_ex against libmtgpu
(oracle/_ref/raytracer_gpu) renders on the GPU and must write the same files
as the reference CLI (oracle/_ref/raytracer)."""
import hashlib
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

PIN = "f9f4551a12c4c73f85c7954ce7e00adebd768798c2471def03df0e97c818ffcb"


def _run(oracle, binary, tmp_path, args, env_extra):
    exe = oracle.HERE / "_ref" / binary
    if not exe.exists():
        pytest.skip(f"{exe} not built")
    out = tmp_path / f"{binary}.bmp"
    env = dict(os.environ, RAYTRACER_NO_PROGRESS="1", **env_extra)
    subprocess.run([str(exe), *args, "--out", str(out)], check=True, env=env, stdout=subprocess.DEVNULL)
    return out.read_bytes()


def test_gpu_cli_reproduces_whitted_pin(oracle, mtlib, tmp_path):
    args = ["--no-pathtrace", "--no-adaptive", "--width", "320", "--height", "180", "--samples", "4", "--depth", "4"]
    data = _run(oracle, "raytracer_gpu", tmp_path, args, {"MT_PRECISION": "fp64"})
    assert hashlib.sha256(data).hexdigest() == PIN


def test_gpu_cli_pathtracer_matches_reference_cli(oracle, mtlib, tmp_path):
    args = ["--width", "160", "--height", "90", "--samples", "4", "--depth", "4"]
    gpu = _run(oracle, "raytracer_gpu", tmp_path, args, {"MT_PRECISION": "fp64"})
    cpu = _run(oracle, "raytracer", tmp_path, args, {})
    assert len(gpu) == len(cpu)
    diff = sum(a != b for a, b in zip(gpu, cpu))
    assert diff <= len(cpu) * 1e-4, f"{diff} bytes differ"


def test_gpu_cli_cpu_backend_switch(oracle, mtlib, tmp_path):
    """MT_BACKEND=cpu routes the wrapped entry points to the reference's own
    code (__real_*): same bytes as the reference CLI."""
    args = ["--no-pathtrace", "--no-adaptive", "--width", "64", "--height", "36", "--samples", "1", "--depth", "2"]
    a = _run(oracle, "raytracer_gpu", tmp_path, args, {"MT_BACKEND": "cpu"})
    b = _run(oracle, "raytracer", tmp_path, args, {})
    assert a == b
