"""Shared small parity cases: (matrix factory, AMGConfig), one per
coarsening / smoother family on the hot path."""

import draugr
from draugr import problems

CASES = {
    "aggregation_jacobi": (lambda: problems.poisson2d(24),
                           draugr.AMGConfig(coarsening=draugr.AggregationCoarsening(0.25),
                                            smoother=draugr.JacobiSmootherType())),
    "hypre_l1jacobi": (lambda: problems.heterogeneous_diffusion_3d(12, seed=3),
                       draugr.hypre_default_config(agg_trunc_factor=0.2,
                                                   smoother=draugr.L1JacobiSmootherType())),
    "default_hmis_l1gs": (lambda: problems.poisson2d(20), draugr.AMGConfig()),
    "pmis_direct_gs": (lambda: problems.poisson3d(10),
                       draugr.AMGConfig(coarsening=draugr.PMISCoarsening(0.25),
                                        smoother=draugr.ColoredGaussSeidelType())),
    "pmis_standard_spai0": (lambda: problems.heterogeneous_diffusion_3d(10, seed=5),
                            draugr.AMGConfig(coarsening=draugr.PMISCoarsening(
                                0.25, draugr.StandardInterpolation()),
                                smoother=draugr.SPAI0SmootherType())),
    "hmis_chebyshev": (lambda: problems.heterogeneous_diffusion_3d(10, seed=7),
                       draugr.AMGConfig(smoother=draugr.ChebyshevSmootherType())),
    "aggregation_ilu0": (lambda: problems.poisson2d(24),
                         draugr.AMGConfig(coarsening=draugr.AggregationCoarsening(0.25),
                                          smoother=draugr.ILU0SmootherType())),
    "hmis_serial_ilu0": (lambda: problems.heterogeneous_diffusion_3d(10, seed=9),
                         draugr.AMGConfig(smoother=draugr.SerialILU0SmootherType())),
    "aggregation_serial_gs": (lambda: problems.poisson2d(24),
                              draugr.AMGConfig(coarsening=draugr.AggregationCoarsening(0.25),
                                               smoother=draugr.SerialGaussSeidelType())),
    "hmis_l1_serial_gs": (lambda: problems.heterogeneous_diffusion_3d(10, seed=11),
                          draugr.AMGConfig(smoother=draugr.L1SerialGaussSeidelType())),
    "aggregation_spai1": (lambda: problems.poisson2d(16),
                          draugr.AMGConfig(coarsening=draugr.AggregationCoarsening(0.25),
                                           smoother=draugr.SPAI1SmootherType())),
    "rs_direct_l1jacobi": (lambda: problems.heterogeneous_diffusion_3d(10, seed=13),
                           draugr.AMGConfig(coarsening=draugr.RSCoarsening(0.25, draugr.DirectInterpolation()),
                                            smoother=draugr.L1JacobiSmootherType())),
    "aniso27_hmis": (lambda: problems.anisotropic_27pt(9, 1e-3),
                     draugr.AMGConfig(coarsening=draugr.HMISCoarsening(
                         0.25, draugr.ExtendedIInterpolation(0.2)),
                         smoother=draugr.L1JacobiSmootherType())),
}
