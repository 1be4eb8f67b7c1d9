"""Run output and checkpoint/resume (``main/data_management.py:5-126``).

``RunData`` / ``ReadData`` keep the reference's call signatures and dataset layout: datasets
``pdf`` (FP32 snapshots of the ghost-inclusive state, as the reference stores them), ``potential``
and ``density`` (FP32, [Nx, n]), ``time`` and ``energy`` (FP64), each with a leading snapshot
axis that grows by one per ``save_data`` call, plus the run-info text file written by
``Reference.info_file`` and parsed by line position in ``ReadData.read_info``.

Storage: HDF5 through h5py when it is importable (the reference's ``.hdf5`` file).  Without
h5py (this image has none) the same datasets go to a directory ``<name>.vlrun/`` holding one
raw little-endian file per dataset (snapshots appended) and ``meta.json`` with each dataset's
dtype, frame shape and frame count; reads memory-map the files, so ``read_specific_time``
touches only the requested snapshot.

Checkpoints (``save_checkpoint`` / ``ReadData.read_checkpoint`` and ``Stepper.resume_from``)
hold the full-precision state, the field, the stepper's clock and histories, so a resumed run
continues bit for bit where the saved one stopped.  The reference has no resume path.
"""
from __future__ import annotations

import json
import os

import numpy as np

try:  # optional: the reference's own container format
    import h5py  # type: ignore
except ImportError:  # pragma: no cover - absent in this image
    h5py = None

_DATASETS = ("pdf", "potential", "density", "time", "energy")


def _host(x):
    """Host NumPy copy of a device array (``.get()``), tensor or array."""
    if hasattr(x, "get"):
        return np.asarray(x.get())
    if hasattr(x, "detach"):
        return x.detach().cpu().numpy()
    return np.asarray(x)


class _RawStore:
    """One raw file per dataset, frames appended; ``meta.json`` holds dtype/shape/count."""

    def __init__(self, path):
        self.path = path
        self.meta_path = os.path.join(path, "meta.json")

    def _meta(self):
        with open(self.meta_path) as fh:
            return json.load(fh)

    def _write_meta(self, meta):
        tmp = self.meta_path + ".tmp"
        with open(tmp, "w") as fh:
            json.dump(meta, fh)
        os.replace(tmp, self.meta_path)

    def create(self, frames):
        os.makedirs(self.path, exist_ok=True)
        meta = {}
        for name, arr in frames.items():
            arr = np.ascontiguousarray(arr)
            with open(os.path.join(self.path, name + ".bin"), "wb") as fh:
                fh.write(arr.astype(arr.dtype.newbyteorder("<"), copy=False).tobytes())
            meta[name] = {"dtype": arr.dtype.str, "shape": list(arr.shape), "count": 1}
        self._write_meta(meta)

    def append(self, frames):
        meta = self._meta()
        for name, arr in frames.items():
            m = meta[name]
            arr = np.ascontiguousarray(arr, dtype=np.dtype(m["dtype"]))
            if list(arr.shape) != m["shape"]:
                raise ValueError(f"{name}: frame shape {arr.shape} != {tuple(m['shape'])}")
            with open(os.path.join(self.path, name + ".bin"), "ab") as fh:
                fh.write(arr.tobytes())
            m["count"] += 1
        self._write_meta(meta)

    def read(self, name, idx=slice(None)):
        m = self._meta()[name]
        mm = np.memmap(os.path.join(self.path, name + ".bin"), dtype=np.dtype(m["dtype"]),
                       mode="r", shape=(m["count"], *m["shape"]))
        return np.array(mm[idx])


class RunData:
    def __init__(self, folder, filename, shape, geometry, time, refs):
        self.write_filename = folder + filename + (".hdf5" if h5py is not None else ".vlrun")
        self.info_name = folder + filename + "_info.txt"
        self.checkpoint_name = folder + filename + "_checkpoint.npz"
        self.shape = shape
        # recreate the run file (main/data_management.py:7-11)
        refs.info_file(self.info_name, geometry, time)

    def create_file(self, distribution, elliptic, density):
        """First snapshot: the initial state, potential and density; time and energy 0
        (``main/data_management.py:13-34``)."""
        frames = {"pdf": _host(distribution).astype(np.float32),
                  "potential": _host(elliptic.potential).astype(np.float32),
                  "density": _host(density).astype(np.float32),
                  "time": np.array(0.0), "energy": np.array(0.0)}
        if h5py is not None:
            s = self.shape
            with h5py.File(self.write_filename, "w") as f:
                f.create_dataset("pdf", data=frames["pdf"][None], chunks=True,
                                 maxshape=(None, *s), dtype="f")
                for name in ("potential", "density"):
                    f.create_dataset(name, data=frames[name][None], chunks=True,
                                     maxshape=(None, s[0], s[1]), dtype="f")
                f.create_dataset("time", data=[0], chunks=True, maxshape=(None,))
                f.create_dataset("energy", data=[0], chunks=True, maxshape=(None,))
        else:
            _RawStore(self.write_filename).create(frames)

    def save_data(self, distribution, elliptic, density, time, field_energy):
        """Append one snapshot (``main/data_management.py:36-51``)."""
        frames = {"pdf": _host(distribution).astype(np.float32),
                  "potential": _host(elliptic.potential).astype(np.float32),
                  "density": _host(density).astype(np.float32),
                  "time": np.array(float(time)), "energy": np.array(float(field_energy))}
        if h5py is not None:
            with h5py.File(self.write_filename, "a") as f:
                for name in _DATASETS:
                    f[name].resize(f[name].shape[0] + 1, axis=0)
                    f[name][-1] = frames[name]
        else:
            _RawStore(self.write_filename).append(frames)

    def save_checkpoint(self, distribution, elliptic, stepper):
        """Full-precision restart point: state (ghosts included), field and potential, the
        stepper's time, dt, step and write counters and its histories."""
        full = distribution.full_array() if hasattr(distribution, "full_array") else distribution.arr
        np.savez(self.checkpoint_name, f=_host(full),
                 E=_host(elliptic.electric_field), phi=_host(elliptic.potential),
                 time=np.array(float(stepper.time)), dt=np.array(float(stepper.dt)),
                 steps=np.array(int(stepper.steps_counter)),
                 write_counter=np.array(int(stepper.write_counter)),
                 time_array=np.asarray(stepper.time_array), field_energy=np.asarray(stepper.field_energy))


class ReadData:
    def __init__(self, folder, filename):
        self.write_filename = folder + filename + (".hdf5" if h5py is not None else ".vlrun")
        self.info_name = folder + filename + "_info.txt"
        self.checkpoint_name = folder + filename + "_checkpoint.npz"

    def _read(self, name, idx=slice(None)):
        if h5py is not None:
            with h5py.File(self.write_filename, "r") as f:
                return f[name][idx]
        return _RawStore(self.write_filename).read(name, idx)

    def read_data(self):
        """(time, pdf, potential, density, energy) of every snapshot."""
        return tuple(self._read(n) for n in ("time", "pdf", "potential", "density", "energy"))

    def read_specific_time(self, idx):
        """(time, pdf, potential) of snapshot ``idx``."""
        return self._read("time", idx), self._read("pdf", idx), self._read("potential", idx)

    def read_potential_only(self, idx_range):
        sl = slice(idx_range[0], idx_range[1])
        return self._read("time", sl), self._read("potential", sl)

    def read_info(self):
        """Geometry, time and reference values from the run-info file, by line position
        (``main/data_management.py:77-126``)."""
        with open(self.info_name) as fh:
            p = fh.readlines()
        order_x = int(float(p[46].split()[3]))
        res_x = int(float(p[34].split()[2]))
        x_low = float(p[37].split()[3])
        x_high = float(p[38].split()[3])
        order_u = int(float(p[47].split()[3]))
        res_u = int(float(p[35].split()[2]))
        u_low = float(p[39].split()[3])
        u_high = float(p[40].split()[3])
        order_v = int(float(p[48].split()[3]))
        res_v = int(float(p[36].split()[2]))
        v_low = int(float(p[41].split()[3]))
        v_high = int(float(p[42].split()[3]))
        final_time = float(p[43].split()[3])
        write_time = float(p[44].split()[4])
        order_time = float(p[49].split()[3])
        n0 = float(p[6].split()[2])
        T0 = float(p[7].split()[2])
        L0 = float(p[8].split()[3])
        orders = np.array([order_x, order_u, order_v])
        resolutions = np.array([res_x, res_u, res_v])
        lows = np.array([x_low, u_low, v_low])
        highs = np.array([x_high, u_high, v_high])
        time_info = np.array([final_time, write_time, order_time])
        refs = np.array([n0, T0, L0])
        return orders, resolutions, lows, highs, time_info, refs

    def read_checkpoint(self):
        with np.load(self.checkpoint_name) as z:
            return {k: z[k] for k in z.files}
