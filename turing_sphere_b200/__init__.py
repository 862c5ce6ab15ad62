"""turing_sphere_b200: B200-native spherical-harmonic transforms and IMEX
reaction-diffusion steps for turing-sphere's .m models, behind a C ABI
(include/turing_sht.h, libturing_sht.so)."""
from .layout import ShtConfig, gaussGrid, gridForLmax, isPowerOfTwo, lmIndex, nlmCalc, validateConfig
from .sht import Device, ShtPlan, requestShtDevice
from .model import (GpuModel, ModelCompileError, ModelGroup, ModelSession, eigenvalues,
                    formatFailure)
from .registry import defaultParams, mModelByKey, mModels, presets
from .noise import seededNoise, seededSpectrum
from .digest import digestOf, relL2

__all__ = ["ShtConfig", "gaussGrid", "gridForLmax", "isPowerOfTwo", "lmIndex", "nlmCalc",
           "validateConfig", "Device", "ShtPlan", "requestShtDevice", "GpuModel", "ModelGroup", "ModelCompileError",
           "ModelSession", "eigenvalues", "formatFailure", "defaultParams", "mModelByKey",
           "mModels", "presets", "seededNoise", "seededSpectrum", "digestOf", "relL2"]
