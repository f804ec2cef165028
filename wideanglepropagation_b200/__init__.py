"""B200-native multislice propagators (Fresnel, angular spectrum, WPM).

Drop-in for the multislice API of ``wide_angle_propagation`` (the reference
package); the work runs in the hand-written sm_100a kernels of ``libwap.so``.
"""
from .propagation import *  # noqa: F401,F403
from .propagation import Plan, get_plan  # noqa: F401
from .lines import *  # noqa: F401,F403
from .potentials import gaussian_potential  # noqa: F401
from .lippmann_schwinger import *  # noqa: F401,F403
from . import physics, synthetic  # noqa: F401

__version__ = "0.1.0"
