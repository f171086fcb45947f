"""Physical constants and the phase convention of the deterministic solver.

Restates ``witwin/channel/constants.py:10-38`` of the reference: the phasor is
``exp(-j*k*d)``, time dependence ``exp(+j*2*pi*f*t)``, the free-space amplitude
``sqrt(P)*lambda/(4*pi*d)`` and polarization is carried as a world-frame
complex 3-vector that is projected onto the receiver polarization last.
"""

from __future__ import annotations

import math

C0 = 299792458.0
MU0 = 4.0e-7 * math.pi
EPS0 = 1.0 / (MU0 * C0 * C0)
ETA0 = MU0 * C0

# The field kernels use the CODATA 2018 values that the reference's complex
# mirrors use (tests/ad/_reference_fields.py:9-11); the difference to EPS0
# above is below 1e-9 relative and never reaches 0.01 dB.
VACUUM_PERMITTIVITY = 8.8541878128e-12
VACUUM_PERMEABILITY = 1.25663706212e-6

PEC_EFFECTIVE_SIGMA_E = 1.0e9

PHASOR = "exp(-j*k*d)"
TIME_DEPENDENCE = "exp(+j*2*pi*f*t)"
FREE_SPACE_AMPLITUDE = "sqrt(tx_power)*wavelength/(4*pi*distance)"
POLARIZATION = "world_cartesian_complex3_then_receiver_projection"

PHASE_CONVENTION = {
    "phasor": PHASOR,
    "time_dependence": TIME_DEPENDENCE,
    "free_space_amplitude": FREE_SPACE_AMPLITUDE,
    "polarization": POLARIZATION,
}

NARROWBAND_FREQUENCY_OFFSET_LAW = "H(f_ref+df) = C(f_ref)*exp(-j*2*pi*df*delay_s)"

# The cost of the narrowband law as published by the reference consumer
# contract (witwin/channel/constants.py:70-75): free-space spreading, the slab
# fringe scale of the material response, and the dispersion the law drops.
NARROWBAND_FREQUENCY_OFFSET_ERROR_LAW = (
    "relative_error = O(df/f_ref) spreading"
    " + O(df/df_fringe) material"
    " + zeroth_order dispersion;"
    " df_fringe = c/(2*Re(sqrt(eps_r))*thickness_m*cos(theta_t))"
)

__all__ = [
    "C0",
    "EPS0",
    "ETA0",
    "FREE_SPACE_AMPLITUDE",
    "MU0",
    "NARROWBAND_FREQUENCY_OFFSET_ERROR_LAW",
    "NARROWBAND_FREQUENCY_OFFSET_LAW",
    "PEC_EFFECTIVE_SIGMA_E",
    "PHASE_CONVENTION",
    "PHASOR",
    "POLARIZATION",
    "TIME_DEPENDENCE",
    "VACUUM_PERMEABILITY",
    "VACUUM_PERMITTIVITY",
]
