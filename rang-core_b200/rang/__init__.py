"""rang — the B200-native w-gridder behind rang-core's gridder API.

`rang._core` is the compiled extension with the reference's Python-level
gridder and weighting functions (`wgridder_vis2dirty_f64`, `imaging_weights`
...), so the reference's own Python modules run on it unchanged.
`rang.gridder` and `rang.weighting` are this library's host-array calls over
it, `rang.wgrid_torch` the persistent device plan and the differentiable
degridder, `rang.fista` and `rang.learned` the solvers, `rang.gram` the
visibility-free Gram operator, and `rang.msv4` / `rang.msv2` the readers.
"""
