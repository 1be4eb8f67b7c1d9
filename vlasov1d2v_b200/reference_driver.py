"""Run the reference's own driver script unchanged on this package.

    python -m vlasov1d2v_b200.reference_driver <reference checkout>/main/main.py [--workdir DIR]

``main/main.py`` of crewsdw/Vlasov1D2V imports its sibling modules by their bare names
(``basis``, ``grid``, ``elliptic``, ``timestep``, ``fluxes``, ``reference``, ``data_management``)
and ``cupy``, ``matplotlib`` and ``pyvista`` (``main/main.py:1-13``).  ``run_driver`` executes the
file as it is, with those names resolved to this package's modules (the same classes and call
signatures), ``cupy`` to ``cupy_compat`` and the two plotting packages to inert stand-ins: the
script's figures and its 3-D render (``main/main.py:96-110``, ``:180-227``) are skipped: the
package has no graphics path.  ``RunData`` writes the run files into the working directory (HDF5 when
``h5py`` is importable, raw per-dataset files otherwise).  The script ends with ``quit()``; the
globals it built (``stepper``, ``f0``, ``e``, ``grids`` ...) are returned.
"""
from __future__ import annotations

import argparse
import contextlib
import os
import sys
import types

_ALIASES = ("basis", "grid", "elliptic", "timestep", "fluxes", "reference", "data_management")


class _Inert:
    """Stand-in for plotting objects: every attribute, call and item assignment is a no-op."""

    def __getattr__(self, name):
        return _Inert()

    def __call__(self, *args, **kwargs):
        return _Inert()

    def __setitem__(self, key, value):
        pass

    def __getitem__(self, key):
        return _Inert()


def _plot_modules():
    mpl = types.ModuleType("matplotlib")
    plt = types.ModuleType("matplotlib.pyplot")
    plt.__getattr__ = lambda name: _Inert()
    mpl.__getattr__ = lambda name: _Inert()
    mpl.pyplot = plt
    pv = types.ModuleType("pyvista")
    pv.__getattr__ = lambda name: _Inert()
    return {"matplotlib": mpl, "matplotlib.pyplot": plt, "pyvista": pv}


@contextlib.contextmanager
def driver_modules():
    """``sys.modules`` with the driver's import names bound to this package (restored on exit)."""
    import importlib

    from . import cupy_compat

    names = list(_ALIASES) + ["cupy", "matplotlib", "matplotlib.pyplot", "pyvista"]
    saved = {k: sys.modules.get(k) for k in names}
    try:
        for k in _ALIASES:
            sys.modules[k] = importlib.import_module(f"vlasov1d2v_b200.{k}")
        sys.modules["cupy"] = cupy_compat
        sys.modules.update(_plot_modules())
        yield
    finally:
        for k, v in saved.items():
            if v is None:
                sys.modules.pop(k, None)
            else:
                sys.modules[k] = v


def run_driver(path, workdir=None):
    """Execute the driver script at ``path`` unchanged; returns its global namespace."""
    path = os.path.abspath(path)
    with open(path) as fh:
        code = compile(fh.read(), path, "exec")
    g = {"__name__": "__main__", "__file__": path}
    cwd = os.getcwd()
    if workdir is not None:
        os.makedirs(workdir, exist_ok=True)
        os.chdir(workdir)
    try:
        with driver_modules():
            try:
                exec(code, g)
            except SystemExit:   # the script ends with quit()
                pass
    finally:
        os.chdir(cwd)
    return g


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("script", help="path of the reference's main/main.py")
    ap.add_argument("--workdir", default=None, help="directory for the run files (default: cwd)")
    args = ap.parse_args(argv)
    g = run_driver(args.script, args.workdir)
    st = g.get("stepper")
    if st is not None:
        print(f"steps {st.steps_counter}, final time {st.time:.6f}, "
              f"last field energy {st.field_energy[-1]:.6e}")


if __name__ == "__main__":
    main()
