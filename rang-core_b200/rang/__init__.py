"""rang — the B200-native w-gridder behind rang-core's gridder API.

`rang._core` is the compiled extension with the reference's Python-level
gridder functions (`wgridder_vis2dirty_f64` ...), `rang.core_wgridder` the
keyword API over it (`vis2dirty`, `dirty_psf`, `dirty2vis`, `fits_image`),
`rang.wgrid_torch` the differentiable degridder and the persistent device
plan, and `rang.fista` plain FISTA through the GPU gridder.
"""
