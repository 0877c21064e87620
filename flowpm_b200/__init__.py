"""flowpm_b200: FlowPM's particle-mesh N-body step on NVIDIA B200.

Drop-in for the ``flowpm`` API of the PM hot path (``linear_field``,
``lpt_init``, ``nbody``, ``cic_paint``, ``cic_readout`` and the
``kernels`` Fourier operators), taking and returning torch CUDA tensors.
All compute runs in hand-written sm_100a CUDA kernels (plus cuFFT) inside
``libflowpm_b200.so``, reached through its C ABI (include/flowpm_b200.h).
"""
from . import _lib  # noqa: F401  (fails loudly if the CUDA library is missing)
from . import cosmology
from . import kernels
from . import tfbackground
from . import tfbackground as background
from . import tfpower
from . import raytracing
from . import io
from .utils import cic_paint, cic_readout, r2c3d, c2r3d, white_noise
from .tfpm import nbody, linear_field, lpt_init
from .pk import power_spectrum
from .batch import BatchRunner, nbody_many
from .stream import NBodyStream, nbody_stream
from ._plans import clear_plans, set_autotune

__version__ = '0.1.0'
