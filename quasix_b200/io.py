"""Density-fitting tensors and evGW results on disk, without PySCF or HDF5.

The reference stores both in HDF5 (h5py / hdf5-rust), which this image does
not have.  The same schema -- group and dataset paths, dtypes, shapes,
attributes and validation -- is kept here in an uncompressed NumPy ``.npz``
archive: every HDF5 dataset ``/a/b/c`` is the array ``a/b/c``, the
attributes of a group are one JSON document under ``<group>/.attrs``, and each
dataset carries a CRC-32 (zlib) in ``.checksums`` that plays the role of the
reference's Fletcher-32 filter.

* ``DFTensorsS24`` / ``DFMetadata``: quasix_core/src/io/df_tensors.rs:108-470
  (``/df_tensors/{metric_2c, cderi_3c, iaP, ijP}`` and ``/metadata``, with
  validate_schema's checks).  ``lpq_from_cderi`` turns the packed Cholesky
  vectors into the RI-normalised lpq [naux, nmo, nmo] of this library on the
  GPU (qx_build_lpq with an identity metric step).
* ``save_evgw_results`` / ``load_evgw_results``: the groups of
  EvGWResult.save_to_hdf5 (quasix/quasix/evgw.py:196-380): ``/metadata``,
  ``/parameters``, ``/results/{qp_energies, z_factors}``,
  ``/results/self_energy``, ``/results/convergence``,
  ``/results/iteration_history/iteration_NNN``, ``/results/properties``.
"""
from __future__ import annotations

import json
import time
import zlib
from dataclasses import asdict, dataclass
from typing import Any, Dict, Optional

import numpy as np

HARTREE_TO_EV = 27.2114
SCHEMA_VERSION = "1.0"


def _crc(a: np.ndarray) -> int:
    return zlib.crc32(np.ascontiguousarray(a).view(np.uint8).reshape(-1)) & 0xFFFFFFFF


def _write_npz(path: str, datasets: Dict[str, np.ndarray], attrs: Dict[str, Dict[str, Any]]) -> None:
    out = {k: np.ascontiguousarray(v) for k, v in datasets.items()}
    for g, a in attrs.items():
        out[f"{g}/.attrs"] = np.frombuffer(json.dumps(a).encode(), dtype=np.uint8)
    out[".checksums"] = np.frombuffer(json.dumps({k: _crc(v) for k, v in datasets.items()}).encode(),
                                      dtype=np.uint8)
    with open(path, "wb") as f:
        np.savez(f, **out)


def _read_npz(path: str):
    with np.load(path, allow_pickle=False) as z:
        files = {k: z[k] for k in z.files}
    sums = json.loads(files.pop(".checksums").tobytes().decode())
    attrs = {}
    for k in [k for k in files if k.endswith("/.attrs")]:
        attrs[k[: -len("/.attrs")]] = json.loads(files.pop(k).tobytes().decode())
    for k, v in files.items():
        if k not in sums:
            raise ValueError(f"dataset {k} has no checksum")
        if _crc(v) != sums[k]:
            raise ValueError(f"checksum mismatch in dataset {k}: the file is corrupt")
    return files, attrs


# ---------------------------------------------------------------------------
# DF tensors (df_tensors.rs)
# ---------------------------------------------------------------------------
@dataclass
class DFMetadata:
    """df_tensors.rs:121-144."""
    naux: int
    nao: int
    nocc: int
    nvir: int
    auxbasis: str = "unknown"
    basis: str = "unknown"
    version: str = SCHEMA_VERSION
    timestamp: Optional[str] = None
    git_commit: Optional[str] = None


@dataclass
class DFTensorsS24:
    """df_tensors.rs:108-119: metric_2c [naux, naux], cderi_3c [naux,
    nao (nao + 1) / 2] (packed lower triangle of each AO pair matrix, row by
    row), iaP [nocc nvir, naux], ijP [nocc nocc, naux]."""
    metric_2c: np.ndarray
    cderi_3c: np.ndarray
    ia_p: np.ndarray
    ij_p: np.ndarray
    metadata: DFMetadata

    def validate_schema(self) -> None:
        """The checks of df_tensors.rs:381-468."""
        m = self.metadata
        naux, nao, nocc, nvir = m.naux, m.nao, m.nocc, m.nvir
        if self.metric_2c.shape != (naux, naux):
            raise ValueError(f"metric_2c shape mismatch: expected ({naux}, {naux}), got {self.metric_2c.shape}")
        asym = float(np.abs(self.metric_2c - self.metric_2c.T).max()) if naux else 0.0
        if asym > 1e-10:
            raise ValueError(f"metric_2c is not symmetric: max asymmetry = {asym}")
        npk = nao * (nao + 1) // 2
        if self.cderi_3c.shape != (naux, npk):
            raise ValueError(f"cderi_3c shape mismatch: expected ({naux}, {npk}), got {self.cderi_3c.shape}")
        if self.ia_p.shape != (nocc * nvir, naux):
            raise ValueError(f"ia_p shape mismatch: expected ({nocc * nvir}, {naux}), got {self.ia_p.shape}")
        if self.ij_p.shape != (nocc * nocc, naux):
            raise ValueError(f"ij_p shape mismatch: expected ({nocc * nocc}, {naux}), got {self.ij_p.shape}")
        for name, a in (("metric_2c", self.metric_2c), ("cderi_3c", self.cderi_3c), ("ia_p", self.ia_p),
                        ("ij_p", self.ij_p)):
            if not np.all(np.isfinite(a)):
                raise ValueError(f"{name} contains NaN or Inf values")
        if m.version != SCHEMA_VERSION:
            raise ValueError(f"Unsupported schema version: {m.version} (expected {SCHEMA_VERSION})")

    def write(self, path: str) -> None:
        self.validate_schema()
        md = asdict(self.metadata)
        if md["timestamp"] is None:
            md["timestamp"] = time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime())
        _write_npz(path, {"df_tensors/metric_2c": np.asarray(self.metric_2c, np.float64),
                          "df_tensors/cderi_3c": np.asarray(self.cderi_3c, np.float64),
                          "df_tensors/iaP": np.asarray(self.ia_p, np.float64),
                          "df_tensors/ijP": np.asarray(self.ij_p, np.float64)},
                   {"metadata": md})

    @classmethod
    def read(cls, path: str) -> "DFTensorsS24":
        files, attrs = _read_npz(path)
        if "metadata" not in attrs:
            raise ValueError("missing /metadata")
        for k in ("metric_2c", "cderi_3c", "iaP", "ijP"):
            if f"df_tensors/{k}" not in files:
                raise ValueError(f"missing /df_tensors/{k}")
        d = cls(files["df_tensors/metric_2c"], files["df_tensors/cderi_3c"], files["df_tensors/iaP"],
                files["df_tensors/ijP"], DFMetadata(**attrs["metadata"]))
        d.validate_schema()
        return d


def unpack_cderi(cderi_3c: np.ndarray, nao: int) -> np.ndarray:
    """[naux, nao (nao + 1) / 2] packed lower triangles -> (uv|P) [nao, nao, naux]."""
    naux = cderi_3c.shape[0]
    il, jl = np.tril_indices(nao)
    out = np.empty((nao, nao, naux))
    out[il, jl, :] = cderi_3c.T
    out[jl, il, :] = cderi_3c.T
    return out


def lpq_from_cderi(df: DFTensorsS24, mo_coeff, device: int = 0) -> np.ndarray:
    """lpq [naux, nmo, nmo] = C^T L_P C of the (already RI-normalised)
    Cholesky vectors, on the GPU (qx_build_lpq with J^-1/2 = I)."""
    from .df import build_lpq
    j3 = unpack_cderi(df.cderi_3c, df.metadata.nao)
    lpq, _ = build_lpq(j3, mo_coeff, metric_inv_sqrt=np.eye(df.metadata.naux), device=device)
    return lpq


# ---------------------------------------------------------------------------
# evGW results (EvGWResult.save_to_hdf5)
# ---------------------------------------------------------------------------
def save_evgw_results(path: str, result: Dict[str, Any], nocc: int, parameters: Optional[Dict[str, Any]] = None,
                      vxc_dft=None, total_time: float = 0.0) -> None:
    """``result`` is the dictionary of run_evgw / evgw (qp_energies, z_factors,
    sigma_x, sigma_c_re, sigma_c_im, converged, n_cycles, final_error,
    iteration_history)."""
    qp = np.asarray(result["qp_energies"], np.float64)
    nmo = qp.shape[0]
    p = dict(parameters or {})
    ds = {"results/qp_energies": qp, "results/z_factors": np.asarray(result["z_factors"], np.float64),
          "results/self_energy/sigma_x": np.asarray(result["sigma_x"], np.float64),
          "results/self_energy/sigma_c_real": np.asarray(result["sigma_c_re"], np.float64),
          "results/self_energy/sigma_c_imag": np.asarray(result["sigma_c_im"], np.float64),
          "results/self_energy/vxc_dft": np.zeros(nmo) if vxc_dft is None else np.asarray(vxc_dft, np.float64)}
    hist = result.get("iteration_history", [])
    if hist:
        ds["results/convergence/energy_history"] = np.array([h["qp_energies"] for h in hist])
        ds["results/convergence/error_history"] = np.array([h["energy_change"] for h in hist])
    attrs = {
        "": {"file_format": "QuasiX-NPZ (schema of QuasiX-HDF5)", "file_version": SCHEMA_VERSION,
             "created_by": "quasix_b200", "creation_date": time.strftime("%Y-%m-%dT%H:%M:%S")},
        "metadata": {"quasix_version": "0.1.0", "timestamp": time.strftime("%Y-%m-%dT%H:%M:%S")},
        "parameters": {"calculation_type": "EvGW"},
        "parameters/convergence": {"energy_tol": p.get("conv_tol", 1e-4), "max_iterations": p.get("max_cycle", 12),
                                   "use_diis": p.get("diis", True), "diis_space": p.get("diis_space", 6)},
        "parameters/frequency": {"grid_type": p.get("freq_int", "ac"), "n_points": p.get("nfreq", 48)},
        "parameters/gw_params": {"damping": p.get("damping", 0.5)},
        "results/convergence": {"converged": bool(result["converged"]), "n_cycles": int(result["n_cycles"]),
                                "final_error": float(result["final_error"])},
        "results/timings": {"total_time": float(total_time)},
    }
    for i, h in enumerate(hist):
        g = f"results/iteration_history/iteration_{i:03d}"
        ds[f"{g}/qp_energies"] = np.asarray(h["qp_energies"], np.float64)
        ds[f"{g}/z_factors"] = np.asarray(h["z_factors"], np.float64)
        attrs[g] = {"cycle": int(h["cycle"]), "energy_change": float(h["energy_change"]),
                    "rms_change": float(h["rms_change"]), "damping_used": float(h["damping_used"]),
                    "converged": bool(h["converged"])}
    if nmo > nocc:
        gap = float(qp[nocc] - qp[nocc - 1])
        attrs["results/properties"] = {"homo_index": nocc - 1, "lumo_index": nocc, "gap": gap,
                                       "gap_eV": gap * HARTREE_TO_EV, "ip": float(-qp[nocc - 1]),
                                       "ip_eV": float(-qp[nocc - 1]) * HARTREE_TO_EV, "ea": float(-qp[nocc]),
                                       "ea_eV": float(-qp[nocc]) * HARTREE_TO_EV}
    _write_npz(path, ds, attrs)


def load_evgw_results(path: str) -> Dict[str, Any]:
    """The saved results as a dictionary with run_evgw's keys, plus
    ``attrs`` (every group's attributes) and ``vxc_dft``."""
    files, attrs = _read_npz(path)
    conv = attrs.get("results/convergence", {})
    out = {"qp_energies": files["results/qp_energies"], "z_factors": files["results/z_factors"],
           "sigma_x": files["results/self_energy/sigma_x"],
           "sigma_c_re": files["results/self_energy/sigma_c_real"],
           "sigma_c_im": files["results/self_energy/sigma_c_imag"],
           "vxc_dft": files["results/self_energy/vxc_dft"], "converged": conv.get("converged"),
           "n_cycles": conv.get("n_cycles"), "final_error": conv.get("final_error"), "attrs": attrs}
    hist = []
    i = 0
    while f"results/iteration_history/iteration_{i:03d}/qp_energies" in files:
        g = f"results/iteration_history/iteration_{i:03d}"
        hist.append(dict(attrs.get(g, {}), qp_energies=files[f"{g}/qp_energies"], z_factors=files[f"{g}/z_factors"]))
        i += 1
    out["iteration_history"] = hist
    props = attrs.get("results/properties")
    if props:
        out.update(ip=props["ip"], ea=props["ea"], gap=props["gap"])
    return out
