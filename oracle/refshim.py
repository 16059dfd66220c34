"""Test infrastructure only: import the UNMODIFIED reference modules from a read-only checkout.

The reference's float focuser imports ``sarpy.io.phase_history.converter`` at module level
(``src/form_image_pfa.py:37``) and the emulator reaches the CPHD through that reader
(``mpfs/host/silicon_emulator.py:217-223``).  sarpy is not installed, so this module puts a stub
package in ``sys.modules`` whose ``open_phase_history`` returns a registered fake reader
(``pfa_b200.synth.FakeReader``) for a synthetic scene.  Nothing in the reference is patched.

Used by ``tests/golden/make_golden.py`` and by CPU tests that pin the oracle against the reference.
It only works where the reference checkout exists (``PFA_REFERENCE_ROOT``, default: a ``reference``
checkout beside this repository); the GPU tests, ``smoke()`` and ``bench.py`` never import it.
"""
from __future__ import annotations

import contextlib
import io
import os
import sys
import types
from pathlib import Path

REF_ROOT = Path(os.environ.get("PFA_REFERENCE_ROOT", Path(__file__).resolve().parents[2] / "reference"))
_READERS: dict[str, object] = {}


def available() -> bool:
    return (REF_ROOT / "mpfs" / "host" / "silicon_emulator.py").is_file()


def register_reader(path: str, reader) -> str:
    """Make ``open_phase_history(path)`` return ``reader``."""
    _READERS[str(path)] = reader
    return str(path)


def _install_sarpy_stub():
    if "sarpy.io.phase_history.converter" in sys.modules:
        return
    names = ["sarpy", "sarpy.io", "sarpy.io.phase_history", "sarpy.io.phase_history.converter"]
    mods = [types.ModuleType(n) for n in names]
    for parent, child in zip(mods[:-1], mods[1:]):
        setattr(parent, child.__name__.rsplit(".", 1)[1], child)

    def open_phase_history(path):
        try:
            return _READERS[str(path)]
        except KeyError:
            raise FileNotFoundError(f"no fake reader registered for {path}") from None

    mods[-1].open_phase_history = open_phase_history
    for n, mo in zip(names, mods):
        sys.modules[n] = mo


_MODS = None


def modules():
    """Return a namespace with the reference modules: ref (form_image_pfa), emu (silicon_emulator),
    fx (fixedpoint), pipe (sar_pipeline), ser (serialize_inputs), grv (gen_resample_vectors), accel,
    mdf (model_detect_fusion)."""
    global _MODS
    if _MODS is not None:
        return _MODS
    if not available():
        raise RuntimeError(f"reference checkout not found at {REF_ROOT}")
    _install_sarpy_stub()
    for sub in ("src", "mpfs/host", "mpfs/fpga/tb"):
        p = str(REF_ROOT / sub)
        if p not in sys.path:
            sys.path.insert(0, p)
    with contextlib.redirect_stdout(io.StringIO()):
        import form_image_pfa as ref          # noqa: E402
        import fixedpoint as fx               # noqa: E402
        import sar_pipeline as pipe           # noqa: E402
        import serialize_inputs as ser        # noqa: E402
        import silicon_emulator as emu        # noqa: E402
        import gen_resample_vectors as grv    # noqa: E402
        import accel                          # noqa: E402
        import model_detect_fusion as mdf     # noqa: E402
    _MODS = types.SimpleNamespace(ref=ref, fx=fx, pipe=pipe, ser=ser, emu=emu, grv=grv, accel=accel, mdf=mdf)
    return _MODS


def emulator_form_image(scene, grid, range_sinc, az_sinc, deci=1, quiet=True):
    """Run the reference ``silicon_emulator.form_image`` unmodified on a synthetic scene."""
    from pfa_b200.synth import FakeReader   # noqa: E402
    m = modules()
    path = register_reader(f"synthetic://{id(scene)}", FakeReader(scene))
    ctx = contextlib.redirect_stdout(io.StringIO()) if quiet else contextlib.nullcontext()
    with ctx:
        return m.emu.form_image(path, deci, grid, range_sinc=range_sinc, az_sinc=az_sinc)


def reference_tables(scene, deci=1):
    from pfa_b200.synth import FakeReader   # noqa: E402
    m = modules()
    rd = FakeReader(scene)
    return m.pipe.prepare_tables(rd, rd.cphd_meta, deci, deci)
