"""Import the reference's own Wilson-fermion modules under the numpy JAX shim.

Test infrastructure only: used by ``make_golden.py`` in a container where the
reference sources are mounted.  The reference package ``__init__`` files pull
in unrelated models (flows, optax), so the packages are registered as empty
namespace stubs whose ``__path__`` points at the reference tree, and only the
modules on the Wilson path are executed:

  jaxqft/fermions/gamma.py, jaxqft/fermions/wilson.py,
  jaxqft/core/hamiltonian.py, jaxqft/core/integrators.py, jaxqft/core/update.py,
  jaxqft/models/su3_ym.py, jaxqft/models/su3_wilson_nf2.py
"""

from __future__ import annotations

import importlib
import os
import sys
import types

SHIM_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_shim")


def load_reference(ref_root: str):
    if not os.path.isdir(os.path.join(ref_root, "jaxqft")):
        raise FileNotFoundError(f"reference tree not found under {ref_root}")
    if SHIM_DIR not in sys.path:
        sys.path.insert(0, SHIM_DIR)
    import jax  # noqa: F401  (the shim)

    def stub(name: str, rel: str):
        mod = types.ModuleType(name)
        mod.__path__ = [os.path.join(ref_root, rel)]
        sys.modules[name] = mod
        return mod

    pkg = stub("jaxqft", "jaxqft")
    core = stub("jaxqft.core", "jaxqft/core")
    ferm = stub("jaxqft.fermions", "jaxqft/fermions")
    models = stub("jaxqft.models", "jaxqft/models")
    testing = stub("jaxqft.testing", "jaxqft/testing")
    pkg.core, pkg.fermions, pkg.models, pkg.testing = core, ferm, models, testing

    ham = importlib.import_module("jaxqft.core.hamiltonian")
    integ = importlib.import_module("jaxqft.core.integrators")
    upd = importlib.import_module("jaxqft.core.update")
    core.HamiltonianModel = ham.HamiltonianModel
    core.Monomial = ham.Monomial
    for n in ("Leapfrog", "MinNorm2", "ForceGradient", "MinNorm4PF4"):
        setattr(core, n, getattr(integ, n))
    core.HMC = upd.HMC

    gamma = importlib.import_module("jaxqft.fermions.gamma")
    wilson = importlib.import_module("jaxqft.fermions.wilson")
    ferm.WilsonDiracOperator = wilson.WilsonDiracOperator
    ferm.build_euclidean_gamma = gamma.build_euclidean_gamma
    ferm.gamma5 = gamma.gamma5
    ferm.check_gamma_algebra = gamma.check_gamma_algebra

    class _SmokeConfig:  # the MCMC smoke suite is not on the path
        pass

    testing.SmokeConfig = _SmokeConfig
    testing.run_nf2_mcmc_smoke_suite = None

    su3_ym = importlib.import_module("jaxqft.models.su3_ym")
    nf2 = importlib.import_module("jaxqft.models.su3_wilson_nf2")
    return types.SimpleNamespace(
        gamma=gamma, wilson=wilson, hamiltonian=ham, integrators=integ, update=upd, su3_ym=su3_ym, nf2=nf2
    )
