"""Checkpoint / restart of long evolutions (the `_temp.mat` restart files of
examples/rydberg_pollution_density_matrix_gpu_restart.jl:151-189, writer `write_data_file`
:238-266).

No MAT-file library is available, so the container is NumPy's ``.npz`` (a zip of ``.npy``
arrays, readable without this package).  Field names follow the reference writer: scalars
and arrays are stored as they are; an MPS (a device ``MPS`` or a list of host site arrays,
the reference's ``collect.(rho)``) is stored site by site as ``<name>/<k>`` (column-major
``[chiL, d, chiR]`` complex128) and restored as a device ``MPS`` (or host sites).  A write
goes to ``<file>.tmp`` first and is renamed into place, so an interrupted write never
replaces the previous checkpoint.
"""
import json
import os

import numpy as np

_MPS_KEY = "__mps__"


def write_data_file(filename, fields):
    """Write ``fields`` (name -> scalar / array / MPS / list of site arrays) to ``filename``."""
    arrays, mps_names = {}, []
    for name, v in fields.items():
        if "/" in name or name == _MPS_KEY:
            raise ValueError("field name %r is reserved" % name)
        sites = None
        if hasattr(v, "sites") and hasattr(v, "dims"):          # device MPS
            sites = v.sites()
        elif isinstance(v, (list, tuple)) and v and all(isinstance(a, np.ndarray) and a.ndim == 3 for a in v):
            sites = list(v)
        if sites is not None:
            mps_names.append(name)
            for k, a in enumerate(sites):
                arrays["%s/%d" % (name, k)] = np.asarray(a, dtype=np.complex128)
        else:
            arrays[name] = np.asarray(v)
    arrays[_MPS_KEY] = np.frombuffer(json.dumps(mps_names).encode(), dtype=np.uint8)
    tmp = filename + ".tmp"
    with open(tmp, "wb") as f:
        np.savez(f, **arrays)
    os.replace(tmp, filename)


def read_data_file(filename, ctx=None, device=True):
    """Read a checkpoint.  MPS fields come back as device ``MPS`` objects on ``ctx`` (the
    default context when None) if ``device``, else as lists of host site arrays; 0-d arrays
    come back as Python scalars."""
    out = {}
    with np.load(filename, allow_pickle=False) as z:
        mps_names = json.loads(bytes(z[_MPS_KEY]).decode())
        for name in z.files:
            if name == _MPS_KEY or "/" in name:
                continue
            a = z[name]
            out[name] = a.item() if a.ndim == 0 else a
        for name in mps_names:
            n = sum(1 for f in z.files if f.startswith(name + "/"))
            sites = [z["%s/%d" % (name, k)] for k in range(n)]
            if device:
                from .core import MPS
                out[name] = MPS.from_sites(sites, ctx)
            else:
                out[name] = sites
    return out
