"""B200-native (sm_100a) SU(3) Wilson-fermion hot path with jaxQFT's API.

The compute path is the in-tree CUDA library ``libwilson_sm100.so``
(``jaxqft_b200/csrc``, C-ABI in ``include/wilson_sm100.h``) driven through
``jaxqft_b200.lib``; ``jaxqft_b200.su3_wilson_nf2.SU3WilsonNf2`` mirrors
``jaxqft.models.su3_wilson_nf2.SU3WilsonNf2`` on torch CUDA tensors, and
``jaxqft_b200.update`` / ``integrators`` / ``hamiltonian`` mirror the HMC hooks
of ``jaxqft.core``.
"""

__version__ = "0.1.0"


def __getattr__(name):
    import importlib

    if name in ("lib", "build", "gamma", "su3_ym", "su3_wilson_nf2", "update", "integrators", "hamiltonian",
                "serving", "wilson", "measurements", "lime", "hmc_run", "hmc_compare", "stats"):
        return importlib.import_module(f".{name}", __name__)
    if name == "SU3WilsonNf2":
        return importlib.import_module(".su3_wilson_nf2", __name__).SU3WilsonNf2
    raise AttributeError(name)
