"""periodfind_b200: periodfind's batched periodograms (Conditional Entropy,
Analysis of Variance, Lomb-Scargle, FPW, box least squares) on NVIDIA B200
(sm_100a).

    from periodfind_b200.gpu import ConditionalEntropy, AOV, LombScargle, FPW
    ce = ConditionalEntropy(n_phase=10, n_mag=10)
    stats = ce.calc(times, mags, periods, period_dts, output="stats")

The classes mirror periodfind.gpu's; results come from hand-written CUDA
kernels behind the C ABI in include/pf.h.  Importing this package does not
load the native library; constructing a GPU class does, and raises if it is
absent or no B200 is visible.
"""

from .results import Periodogram, Statistics

__all__ = ["Statistics", "Periodogram", "ConditionalEntropy", "AOV", "LombScargle", "FPW",
           "BoxLeastSquares", "gpu"]
__version__ = "0.1.0"


def __getattr__(name):
    if name in ("ConditionalEntropy", "AOV", "LombScargle", "FPW", "BoxLeastSquares", "gpu"):
        import importlib

        gpu = importlib.import_module(__name__ + ".gpu")
        return gpu if name == "gpu" else getattr(gpu, name)
    raise AttributeError(name)
