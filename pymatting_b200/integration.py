"""Switch an imported PyMatting to this package's GPU path.

PyMatting's subpackages re-export functions under their submodules' names
(``pymatting/laplacian/__init__.py:1-7``, ``pymatting/solver/__init__.py:1-2``,
``pymatting/preconditioner/__init__.py:1-3``, ``pymatting/alpha/__init__.py``),
so ``pymatting.laplacian.cf_laplacian`` is the *function*, and the modules
that use a function bound it by ``from ... import`` when they were imported
(``pymatting/alpha/estimate_alpha_cf.py:1-5`` binds ``cf_laplacian``,
``trimap_split``, ``cg``, ``ichol``). Replacing a function therefore means
rebinding every name that refers to it, in every loaded ``pymatting``
module. ``install`` does exactly that: for each replaced function it finds
the original in its defining module (through ``sys.modules``, not through
the shadowed package attribute) and rebinds every attribute of every loaded
``pymatting*`` module that is that object.

    import pymatting
    import pymatting_b200.integration
    pymatting_b200.integration.install()      # pymatting.cg is now the GPU cg

Nothing of PyMatting is edited on disk; ``uninstall`` restores the bindings.
"""

import sys

__all__ = ["HOT_PATH", "NEXT_ROWS", "install", "uninstall", "replacements"]

# (defining module, name): the closed-form alpha hot path.
HOT_PATH = [
    ("pymatting.laplacian.cf_laplacian", "cf_laplacian"),
    ("pymatting.laplacian.laplacian", "make_linear_system"),
    ("pymatting.solver.cg", "cg"),
    ("pymatting.solver.callback", "CounterCallback"),
    ("pymatting.solver.callback", "ProgressCallback"),
    ("pymatting.preconditioner.jacobi", "jacobi"),
    ("pymatting.preconditioner.vcycle", "vcycle"),
    ("pymatting.preconditioner.ichol", "ichol"),
    ("pymatting.preconditioner.ichol", "CholeskyDecomposition"),
    ("pymatting.alpha.estimate_alpha_cf", "estimate_alpha_cf"),
    ("pymatting.util.util", "trimap_split"),
    ("pymatting.util.util", "sanity_check_image"),
]

# The paths built next to it (other Laplacians and estimators, foreground
# estimation, cutout and image files).
NEXT_ROWS = [
    ("pymatting.laplacian.lkm_laplacian", "lkm_laplacian"),
    ("pymatting.laplacian.uniform_laplacian", "uniform_laplacian"),
    ("pymatting.laplacian.rw_laplacian", "rw_laplacian"),
    ("pymatting.laplacian.lbdm_laplacian", "lbdm_laplacian"),
    ("pymatting.laplacian.knn_laplacian", "knn_laplacian"),
    ("pymatting.alpha.estimate_alpha_lkm", "estimate_alpha_lkm"),
    ("pymatting.alpha.estimate_alpha_knn", "estimate_alpha_knn"),
    ("pymatting.alpha.estimate_alpha_lbdm", "estimate_alpha_lbdm"),
    ("pymatting.alpha.estimate_alpha_rw", "estimate_alpha_rw"),
    ("pymatting.foreground.estimate_foreground_ml", "estimate_foreground_ml"),
    ("pymatting.foreground.estimate_foreground_cf", "estimate_foreground_cf"),
    ("pymatting.cutout.cutout", "cutout"),
    ("pymatting.util.util", "load_image"),
    ("pymatting.util.util", "save_image"),
    ("pymatting.util.util", "stack_images"),
    ("pymatting.util.util", "blend"),
]

_saved = []     # (module, attribute, original object) of every rebinding


def replacements(include_next=True):
    """``{(defining module, name): replacement}`` for the rows to switch."""
    import pymatting_b200 as b200
    rows = HOT_PATH + (NEXT_ROWS if include_next else [])
    return {(mod, name): getattr(b200, name) for mod, name in rows}


def install(include_next=True, modules=None):
    """Rebind PyMatting's functions to this package's, in every loaded
    ``pymatting*`` module (``modules``: a name -> module mapping to use
    instead of ``sys.modules``). Returns the number of rebound names.
    Rows whose defining module is not loaded are skipped."""
    mods = sys.modules if modules is None else modules
    table = {}
    for (mod, name), new in replacements(include_next).items():
        m = mods.get(mod)
        if m is None or not hasattr(m, name):
            continue
        old = getattr(m, name)
        if old is not new:
            table[id(old)] = (old, new)
    count = 0
    for mname in sorted(k for k in list(mods) if k == "pymatting" or k.startswith("pymatting.")):
        m = mods[mname]
        if m is None:
            continue
        for attr, val in list(vars(m).items()):
            hit = table.get(id(val))
            if hit is not None and hit[0] is val:
                _saved.append((m, attr, val))
                setattr(m, attr, hit[1])
                count += 1
    return count


def uninstall():
    """Restore every binding ``install`` changed."""
    while _saved:
        m, attr, val = _saved.pop()
        setattr(m, attr, val)
