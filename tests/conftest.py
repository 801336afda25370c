"""Test configuration: the ``gpu`` marker and import paths.

Tests marked ``gpu`` need a CUDA device and the built ``libshtb200.so``; all
others run on CPU only.
"""
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT, ROOT / "shtnskit.jl_b200"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built CUDA library")
