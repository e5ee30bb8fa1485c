"""Run CerebroSim's own driver scripts (validate.py, and vessel.py's geometry) unmodified on this package.

The reference's scripts import `warp` at module top and the solver as the sibling module `lbm` (validate.py:26-30,
vessel.py:26). `install(reference_dir)` prepares an interpreter so that `import validate` there runs on the B200
path:

- `lbm` is `cerebrosim_b200.lbm` (the drop-in solver module);
- `warp` is a small stand-in with what those scripts call outside the kernels this package replaces: `init`,
  `synchronize` (torch.cuda.synchronize), `get_preferred_device`, the `kernel` / `func` / `constant` decorators
  (identity: the reference's Warp kernels are defined but never launched), placeholders for every type name their
  signatures use (`vec3`, `array`, `array3d`, ...) and a `launch` that raises, naming the replacement;
- the reference's `vessel` module is imported from `reference_dir` and its `sdf_grid` (the Warp kernel k_sdf,
  vessel.py:183-245) is routed to `cerebrosim_b200.vessel.sdf_grid`, which returns the same (array, origin).

simulate.py's `ArterySolver` and its sampling loop launch Warp kernels of their own (k_flux, k_bc, k_gather); their
replacements are `cerebrosim_b200.simulate.ArterySolver` and `run_beats`, so `load("simulate")` also sets
`simulate.ArterySolver` to this package's.
"""
import importlib
import math
import sys
import types

_REPLACED = ("lbm", "warp", "vessel", "validate", "simulate")


class _Type:
    """A Warp type name in a signature: callable (wp.array(dtype=...), wp.vec3(...)) and subscriptable."""

    def __init__(self, name):
        self.name = name

    def __call__(self, *a, **k):
        return self

    def __getitem__(self, key):
        return self

    def __repr__(self):
        return f"warp.{self.name} (stand-in)"


def _launch(*a, **k):
    raise NotImplementedError("a reference Warp kernel was launched: this package replaces it (k_step / k_clock: "
                              "cerebrosim_b200.lbm.Solver; k_sdf: cerebrosim_b200.vessel.sdf_grid; k_flux / k_bc: "
                              "cerebrosim_b200.simulate.ArterySolver; k_gather: cerebrosim_b200.simulate.Probes)")


def warp_module():
    """The `warp` stand-in module."""
    import torch

    wp = types.ModuleType("warp")
    wp.__doc__ = "Stand-in for NVIDIA Warp when CerebroSim's scripts run on cerebrosim_b200 (cerebrosim_b200.refshim)."
    wp.init = lambda: None
    wp.synchronize = lambda: torch.cuda.synchronize() if torch.cuda.is_available() else None
    wp.get_preferred_device = lambda: "cuda:0"
    wp.kernel = lambda f=None, **k: f if f is not None else (lambda g: g)
    wp.func = lambda f=None, **k: f if f is not None else (lambda g: g)
    wp.constant = lambda x: x
    wp.set_module_options = lambda *a, **k: None
    wp.launch = _launch
    wp.pi = math.pi
    wp.types = types.SimpleNamespace(vector=lambda length, dtype: _Type(f"vector{length}"))
    # every other name (vec3, array, array3d, uint64, Mesh, ...) is a type placeholder: it appears only in the
    # signatures and bodies of kernels that are never launched
    wp.__getattr__ = lambda name: _Type(name)
    return wp


def install(reference_dir):
    """Make `import validate` / `import vessel` in this interpreter load the reference's unmodified files from
    reference_dir, running on this package. Returns the sys.modules entries it replaced (for `uninstall`)."""
    from . import lbm
    from . import vessel as ours

    saved = {k: sys.modules.get(k) for k in _REPLACED}
    sys.modules["lbm"] = lbm
    sys.modules["warp"] = warp_module()
    if reference_dir not in sys.path:
        sys.path.insert(0, reference_dir)
    for k in ("vessel", "validate", "simulate"):
        sys.modules.pop(k, None)
    vessel = importlib.import_module("vessel")

    def sdf_grid(g, dx, lo=None, hi=None, device=None):
        # vessel.sdf_grid's signature and return value (vessel.py:230-245): the field on the GPU, read back
        return ours.sdf_grid(g, dx, lo, hi, device=device)

    vessel.sdf_grid = sdf_grid
    return saved


def load(name):
    """Import one of the reference's scripts after `install` (simulate.ArterySolver replaced)."""
    mod = importlib.import_module(name)
    if name == "simulate":
        from . import simulate as ours
        mod.ArterySolver = ours.ArterySolver
    return mod


def uninstall(saved):
    """Restore the sys.modules entries `install` replaced."""
    for k, v in saved.items():
        if v is None:
            sys.modules.pop(k, None)
        else:
            sys.modules[k] = v
