"""Drop-in replacement of the reference package bvh_diff_gaussian_rasterization
(diff-gaussian-rasterization/bvh_diff_gaussian_rasterization/__init__.py), backed by the
sm_100a kernels of libgvc.so.

Public surface kept as in the reference: rasterize_gaussians, _RasterizeGaussians,
GaussianRasterizationSettings, GaussianRasterizer (build_bvh, forward, intersect),
cpu_deep_copy_tuple.  Gradients come back in the shapes of the inputs.
"""
from typing import NamedTuple

import torch
import torch.nn as nn

from . import _C


def cpu_deep_copy_tuple(input_tuple):
    """__init__.py:7-12 of the reference."""
    copied_tensors = [item.cpu().clone() if isinstance(item, torch.Tensor) else item for item in input_tuple]
    return tuple(copied_tensors)


def rasterize_gaussians(means3D, scales, rotations, values, weights, raster_settings):
    """__init__.py:15-30 of the reference."""
    return _RasterizeGaussians.apply(means3D, scales, rotations, values, weights, raster_settings)


class _RasterizeGaussians(torch.autograd.Function):
    """__init__.py:33-140 of the reference: forward saves the same eight tensors, backward
    returns five gradients and None for the settings."""

    @staticmethod
    def forward(ctx, means3D, scales, rotations, values, weights, raster_settings):
        vmin = raster_settings.volume_mins
        vmax = raster_settings.volume_maxes
        cells, cell_weights, conics = _C.rasterize_gaussians(
            means3D, scales, rotations, values, weights, raster_settings.scale_modifier,
            vmin[0], vmin[1], vmin[2], vmax[0], vmax[1], vmax[2], raster_settings.bg,
            raster_settings.use_gaussian_bvh, raster_settings.debug)
        ctx.raster_settings = raster_settings
        ctx.save_for_backward(means3D, scales, rotations, values, weights, cells, cell_weights, conics)
        return cells, cell_weights

    @staticmethod
    def backward(ctx, grad_out_cells, grad_out_cell_weights):
        rs = ctx.raster_settings
        means3D, scales, rotations, values, weights, cells, cell_weights, conics = ctx.saved_tensors
        vmin, vmax = rs.volume_mins, rs.volume_maxes
        if grad_out_cells is None:
            grad_out_cells = torch.zeros_like(cells)
        if grad_out_cell_weights is None:
            grad_out_cell_weights = torch.zeros_like(cell_weights)
        g_means, g_scales, g_rots, g_values, g_weights = _C.rasterize_gaussians_backward(
            means3D, scales, rotations, conics, values, weights, cells, cell_weights, rs.scale_modifier,
            vmin[0], vmin[1], vmin[2], vmax[0], vmax[1], vmax[2], rs.bg,
            grad_out_cells.contiguous(), grad_out_cell_weights.contiguous(), rs.use_gaussian_bvh, rs.debug)
        return (g_means.view_as(means3D), g_scales.view_as(scales), g_rots.view_as(rotations),
                g_values.view_as(values), g_weights.view_as(weights), None)


class GaussianRasterizationSettings(NamedTuple):
    volume_mins: tuple
    volume_maxes: tuple
    cell_count: int
    bg: float
    scale_modifier: float
    use_gaussian_bvh: bool
    debug: bool


class GaussianRasterizer(nn.Module):
    """__init__.py:153-229 of the reference."""

    def __init__(self, raster_settings):
        super().__init__()
        self.raster_settings = raster_settings

    def build_bvh(self, samples, force_debug=False, use_gaussian_bvh=False):
        if force_debug:
            _C.build_bvh(samples, True, use_gaussian_bvh)
        else:
            _C.build_bvh(samples, self.raster_settings.debug, use_gaussian_bvh)

    def forward(self, means3D, scales=None, rotations=None, values=None, weights=None, debug=False):
        raster_settings = self.raster_settings._replace(debug=debug) if debug else self.raster_settings
        if scales is None or rotations is None:
            raise Exception("Please provide scale/rotation pair!")
        if values is None:
            raise Exception("Please provide scalar values for each Gaussian!")
        if weights is None:
            raise Exception("Please provide scalar weights for each Gaussian!")
        return rasterize_gaussians(means3D, scales, rotations, values, weights, raster_settings)

    def intersect(self, means3D, scales=None, rotations=None, debug=False):
        # The reference's intersect (__init__.py:207-229) calls a function that is not
        # defined anywhere; it raises the same NameError here.
        if scales is None or rotations is None:
            raise Exception("Please provide scale/rotation pair!")
        raise NameError("name 'intersect_gaussians' is not defined")
