"""Learned preconditioner: a U-Net that maps [gradient, illumination, Vp,
Vs] to a Vs update direction, trained on update pairs that the plain
illumination-preconditioned L-BFGS inversion generates on seeded synthetic
models, and used inside an inversion whose line search accepts a learned
step only if it lowers the misfit (plain L-BFGS is the fallback).

The network runs on the library's own tcgen05 convolution kernels
(include/stfwi_nn.h); there is no framework fallback.
"""
from .unet import UNet, LAYERS, padded_shape  # noqa: F401
