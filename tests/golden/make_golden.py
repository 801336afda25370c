"""Convert the reference's SHTns 3.7 golden vectors for the transform hot path into
``shtns37_hotpath.npz`` (plus a JSON sidecar with each fixture's configuration).

The reference ships the fixtures as little-endian binaries with a TOML manifest
(``test/fixtures/shtns37/manifest.toml``; loader ``test/parity/shtns37_fixtures.jl:10-30``).
Coefficients are in SHTns packed LM order (``src/layout.jl:143-150``) and are
unpacked here to the dense ``(lmax+1, mmax+1[, nfields])`` layout. Fields keep
the ``(nlat, nphi[, nfields])`` shape of the Julia arrays.

Usage (needs the reference checkout, read-only; its root is a required argument)::

    python tests/golden/make_golden.py <path to the SHTnsKit.jl checkout>

The output is committed so that tests run without the reference present.
"""
from __future__ import annotations

import json
import sys
import tomllib
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))
from oracle import sht_oracle as so  # noqa: E402

HOT_PATH_IDS = [
    "scalar_real_full_gauss_f64",
    "scalar_batch",
    "analysis_scalar_full",
    "sphtor_full_f32",
    "sphtor_batch",
    "analysis_sphtor_full",
    "qst_full",
    "analysis_qst_full",
]


def read_payload(root: Path, p: dict) -> np.ndarray:
    raw = (root / p["file"]).read_bytes()
    et = p["eltype"]
    shape = tuple(p["shape"])
    if et == "float64":
        v = np.frombuffer(raw, dtype="<f8")
    elif et == "complex64":          # SHTns manifest: a pair of float64 per element
        r = np.frombuffer(raw, dtype="<f8")
        v = r[0::2] + 1j * r[1::2]
    elif et == "float32":
        v = np.frombuffer(raw, dtype="<f4").astype(np.float64)
    elif et == "complex32":
        r = np.frombuffer(raw, dtype="<f4").astype(np.float64)
        v = r[0::2] + 1j * r[1::2]
    else:
        raise ValueError(et)
    return np.reshape(v, shape, order="F")


def main(ref_root: str) -> None:
    fx_root = Path(ref_root) / "test" / "fixtures" / "shtns37"
    manifest = tomllib.loads((fx_root / "manifest.toml").read_text())
    arrays: dict[str, np.ndarray] = {}
    meta: dict[str, dict] = {}
    for fx in manifest["fixture"]:
        fid = fx["id"]
        if fid not in HOT_PATH_IDS:
            continue
        keys = ("capability", "grid", "norm", "cs_phase", "real_norm", "precision", "lmax", "mmax",
                "mres", "ltr", "nlat", "nphi", "atol", "rtol")
        meta[fid] = {k: fx[k] for k in keys if k in fx}
        meta[fid]["direction"] = fx.get("direction", "synthesis")
        cfg = so.create_gauss_config(fx["lmax"], fx["nlat"], mmax=fx["mmax"], mres=fx["mres"],
                                     nlon=fx["nphi"], norm=fx["norm"], cs_phase=fx["cs_phase"],
                                     real_norm=fx["real_norm"])
        names = []
        for p in fx["payload"]:
            v = read_payload(fx_root, p)
            name = p["name"]
            if name in ("coefficients", "S", "T", "Q"):
                if v.ndim == 1:
                    v = so.unpack_lm(cfg, v)
                else:
                    v = np.stack([so.unpack_lm(cfg, v[:, k]) for k in range(v.shape[1])], axis=2)
            arrays[f"{fid}/{name}"] = v
            names.append(name)
        meta[fid]["payloads"] = names
    np.savez_compressed(HERE / "shtns37_hotpath.npz", **arrays)
    (HERE / "shtns37_hotpath.json").write_text(json.dumps(meta, indent=1, sort_keys=True) + "\n")
    print(f"wrote {len(meta)} fixtures, {len(arrays)} arrays")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: python tests/golden/make_golden.py <path to the SHTnsKit.jl checkout>")
    main(sys.argv[1])
