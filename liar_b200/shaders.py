"""Shaders of the scene API (``liar.shaders``, src/liar/shaders/): parameters only; the BSDFs
themselves run on the GPU (liar_b200/csrc/render_dev.cuh)."""
from __future__ import annotations

from .spectra import Spectrum
from .textures import Constant


class MicrofacetDistribution:
    kind = 0


class MicrofacetBeckmann(MicrofacetDistribution):
    kind = 0  # shaders/microfacet_beckmann.cpp


class MicrofacetTrowbridgeReitz(MicrofacetDistribution):
    kind = 1  # GGX, shaders/microfacet_trowbridge_reitz.cpp


class Shader:
    pass


class Lambert(Shader):
    def __init__(self, diffuse=None):
        self.diffuse = diffuse if diffuse is not None else Constant(1.0)


class Unshaded(Shader):
    """Pure emitter: emission() returns the colour, no BSDF (shaders/unshaded.cpp)."""

    def __init__(self, colour=None):
        self.colour = colour if colour is not None else Constant(1.0)


class Sum(Shader):
    """Sum of shaders (shaders/sum.cpp). Supported on the GPU: at most one BSDF component plus
    Unshaded emitters."""

    def __init__(self, children=()):
        self.children = list(children)


class Mirror(Shader):
    def __init__(self, reflectance=None):
        self.reflectance = reflectance if reflectance is not None else Constant(1.0)


class Conductor(Shader):
    def __init__(self, refractionIndex=None, absorptionCoefficient=None):
        self.refractionIndex = refractionIndex if refractionIndex is not None else Constant(1.0)
        self.absorptionCoefficient = absorptionCoefficient if absorptionCoefficient is not None else Constant(0.0)
        self.reflectance = Constant(1.0)


class CookTorrance(Shader):
    def __init__(self, refractionIndex=None, absorptionCoefficient=None):
        self.refractionIndex = refractionIndex if refractionIndex is not None else Constant(1.0)
        self.absorptionCoefficient = absorptionCoefficient if absorptionCoefficient is not None else Constant(1.0)
        self.reflectance = Constant(1.0)
        self.roughnessU = Constant(0.0)
        self.roughnessV = Constant(0.0)
        self.mdf = MicrofacetBeckmann()
        self.numberOfSamples = 1

    @property
    def roughness(self):
        return self.roughnessU

    @roughness.setter
    def roughness(self, value):
        self.roughnessU = self.roughnessV = value


class Dielectric(Shader):
    def __init__(self, innerRefractionIndex=None, outerRefractionIndex=None):
        self.innerRefractionIndex = innerRefractionIndex if innerRefractionIndex is not None else Constant(1.5)
        self.outerRefractionIndex = outerRefractionIndex if outerRefractionIndex is not None else Constant(1.0)
        self.reflectance = Constant(1.0)
        self.transmittance = Constant(1.0)


class Walter(Dielectric):
    def __init__(self, innerRefractionIndex=None, outerRefractionIndex=None):
        super().__init__(innerRefractionIndex, outerRefractionIndex)
        self.roughnessU = Constant(0.0)
        self.roughnessV = Constant(0.0)
        self.mdf = MicrofacetTrowbridgeReitz()
        self.numberOfSamples = 1

    @property
    def roughness(self):
        return self.roughnessU

    @roughness.setter
    def roughness(self, value):
        self.roughnessU = self.roughnessV = value
