"""Material records (reference: flatworld/materials/materialsclass.py:5-47).

The constitutive laws themselves run on the GPU (csrc/fw_device.cuh):
``Elastic`` is St-Venant-Kirchhoff on the Green-Lagrange strain, ``HyperElastic``
the compressible NeoHookean law, ``MisesPlastic`` J2 radial return with linear
isotropic hardening.
"""

from .definitions import MaterialType


class Elastic:
    def __init__(self, E, nu, rho):
        self.type = MaterialType.ELASTIC
        self.E = E
        self.nu = nu
        self.rho = rho

    def getRepresentativeModulus(self):
        return self.E


class HyperElastic:
    def __init__(self, E, nu, rho):
        self.type = MaterialType.NEOHOOKEAN
        self.E = E
        self.nu = nu
        self.rho = rho

    def getRepresentativeModulus(self):
        return self.E


class MisesPlastic:
    """J2 von Mises plasticity with linear isotropic hardening H."""

    def __init__(self, E, nu, rho, sigma_y, H=0.0):
        self.type = MaterialType.MISES
        self.E = E
        self.nu = nu
        self.rho = rho
        self.sigma_y = sigma_y
        self.H = H

    def getRepresentativeModulus(self):
        return self.E


# Names used by the reference for the NeoHookean and J2 laws in prose.
NeoHookean = HyperElastic
J2 = MisesPlastic


class SolidProp:
    """reference: flatworld/solidprop.py:1-6"""

    def __init__(self, mat):
        self.mat = mat

    def getMaterial(self):
        return self.mat
