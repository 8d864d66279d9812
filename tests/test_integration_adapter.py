"""The reference-side adapter (splatkit-ios_b200/integration/CudaSplatRenderer.h) compiles against
the reference engine's own SplatRenderer interface and links against the library (CPU only).

It needs the reference's headers, which exist only where the reference tree is mounted; the test
skips elsewhere. The location of its `packages` directory is SPLATKIT_REFERENCE, else the one the
oracle build recorded in oracle/_ref/reference_packages when it compiled the reference's C++.
"""
from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def _packages() -> Path:
    env = os.environ.get("SPLATKIT_REFERENCE")
    if env:
        return Path(env)
    recorded = ROOT / "oracle" / "_ref" / "reference_packages"
    return Path(recorded.read_text().strip()) if recorded.exists() else Path("reference-not-found")


PACKAGES = _packages()
LIB_DIR = ROOT / "splatkit-ios_b200"

MAIN = r"""
#include "CudaSplatRenderer.h"
#include <cstdio>
int main() {
  // No device here: construction fails softly and every verb reports failure.
  splatkit::CudaSplatRenderer r(0, 64, 48);
  splatkit::SplatRenderer& base = r;
  splat::SplatCloud cloud;
  splatkit::SplatRenderer::Frame frame;
  frame.orderSource = splatkit::SplatRenderer::OrderSource::gpu;
  const bool ok = base.uploadWorld(cloud, 0) || base.draw(frame) || base.world().has_value();
  std::printf("ready=%d ok=%d extent=%ux%u sorts=%d lod=%d\n", base.ready() ? 1 : 0, ok ? 1 : 0,
              base.drawExtent().width, base.drawExtent().height, base.sortsOnGpu() ? 1 : 0,
              base.selectsLodOnGpu() ? 1 : 0);
  return 0;
}
"""


@pytest.mark.skipif(not (PACKAGES / "splatkit-engine" / "include").is_dir(),
                    reason="the reference engine headers are not mounted here")
@pytest.mark.skipif(shutil.which("g++") is None, reason="no g++")
def test_adapter_builds_against_the_reference_interface(tmp_path):
    lib = LIB_DIR / "libsplatkit_b200.so"
    if not lib.exists():
        pytest.skip("libsplatkit_b200.so is not built")
    src = tmp_path / "main.cpp"
    src.write_text(MAIN)
    exe = tmp_path / "adapter"
    cmd = ["g++", "-std=c++20", "-O1", "-Wall", "-Werror", "-Wno-unused-private-field",
           f"-I{PACKAGES / 'splat-core' / 'include'}", f"-I{PACKAGES / 'splatkit-engine' / 'include'}",
           f"-I{ROOT / 'include'}", f"-I{LIB_DIR / 'integration'}", str(src), "-o", str(exe),
           f"-L{LIB_DIR}", "-lsplatkit_b200", f"-Wl,-rpath,{LIB_DIR}"]
    build = subprocess.run(cmd, capture_output=True, text=True)
    assert build.returncode == 0, build.stderr[-4000:]
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120,
                         env={**os.environ, "CUDA_VISIBLE_DEVICES": ""})
    assert run.returncode == 0, run.stderr
    assert run.stdout.strip() == "ready=0 ok=0 extent=64x48 sorts=1 lod=1"
