"""Physical constants and the internal unit system.

Energies inside the hot path are in the reference's internal unit,
amu * Angstrom^2 / ps^2, so that numbers can be compared with the reference's
own energy routines without conversion. The constants and the derived
conversion factors are restated from src/constants.h:50-60 and
src/constants.c:137-175 of the reference.
"""
import math

ANGSTROM = 1e-10
PICO_SECOND = 1e-12
ATOMIC_MASS_UNIT = 1.6605402e-27          # kg
ELECTRONIC_CHARGE_UNIT = 1.60217733e-19   # C
MOLAR_GAS_CONSTANT = 8.314464919          # J/(mol K)
BOLTZMANN_CONSTANT = 1.380650324e-23      # J/K
AVOGADRO_CONSTANT = 6.0221419947e23       # 1/mol
ELECTRIC_CONSTANT = 8.8541878176e-12      # C^2/(N m^2)

# derived (src/constants.c:147-172)
ENERGY_CONVERSION_FACTOR = ATOMIC_MASS_UNIT * ANGSTROM ** 2 / PICO_SECOND ** 2
PRESSURE_CONVERSION_FACTOR = ATOMIC_MASS_UNIT / (ANGSTROM * PICO_SECOND ** 2)
K_B = BOLTZMANN_CONSTANT / ENERGY_CONVERSION_FACTOR
COULOMBIC_CONVERSION_FACTOR = (ELECTRONIC_CHARGE_UNIT ** 2
                               / (4.0 * math.pi * ELECTRIC_CONSTANT * ANGSTROM
                                  * ENERGY_CONVERSION_FACTOR))
ENERGY_TO_KELVIN = ENERGY_CONVERSION_FACTOR * AVOGADRO_CONSTANT / MOLAR_GAS_CONSTANT
KELVIN_TO_ENERGY = MOLAR_GAS_CONSTANT / (ENERGY_CONVERSION_FACTOR * AVOGADRO_CONSTANT)
ENERGY_TO_KJ_PER_MOL = ENERGY_CONVERSION_FACTOR * AVOGADRO_CONSTANT / 1000.0

# MC defaults of the reference (src/input.c:345-368)
ENERGY_OVERLAP_CRITERIA = 1.0e7
MINIMUM_ROSENBLUTH_FACTOR = 1.0e-150


def beta(temperature_K: float) -> float:
    """1/(k_B T) in inverse internal energy units."""
    return 1.0 / (K_B * temperature_K)


def pressure_to_internal(p_pa: float) -> float:
    return p_pa / PRESSURE_CONVERSION_FACTOR
