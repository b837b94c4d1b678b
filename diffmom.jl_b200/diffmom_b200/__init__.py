"""diffmom_b200 -- B200 library for DiffMoM.jl's dense surface-EFIE hot path.

Host-side mirror of the Julia API (mesh generators, RWG construction and the
EFIE / solver / far-field entry points) over the C ABI of libdiffmom_b200.so.
"""
from .mesh import (TriMesh, make_rect_plate, make_circular_plate, make_icosphere,
                   make_perturbed_ellipsoid, triangle_area, triangle_areas, triangle_centers,
                   nvertices, ntriangles)
from .rwg import RWGData, build_rwg, rwg_centers, basis_triangles
from .api import (EFIEDevice, assemble_Z_efie, matrixfree_efie_operator, MatrixFreeEFIEOperator,
                  PlaneWaveExcitation, make_plane_wave, assemble_plane_wave, assemble_excitation,
                  DipoleExcitation, LoopExcitation, make_dipole, make_loop, assemble_dipole,
                  assemble_loop, PatternFeedExcitation, make_pattern_feed, make_analytic_dipole_pattern_feed,
                  assemble_pattern_feed,
                  assemble_multiple_excitations, build_nearfield_preconditioner, NearFieldOperator,
                  NearFieldAdjointOperator, solve_gmres_adjoint, solve_adjoint_rhs, PatchPartition, PatchMass,
                  precompute_patch_mass, gradient_impedance,
                  solve_gmres, solve_forward, solve_scattering, ScatteringResult, SphGrid,
                  monostatic_rcs_sweep, MonostaticResult, BatchSurface, BatchResult,
                  SurfaceBatch, solve_surfaces,
                  make_sph_grid, phi_cut_grid, compute_farfield, bistatic_rcs, backscatter_rcs,
                  C0_DEFAULT, ETA0_DEFAULT, tune_report)
from .learned import train_learned_network, training_bodies, load_default_network
from .aca import (ClusterNode, ClusterTree, build_cluster_tree, cluster_tree_resource_bounds, aca_block_tasks,
                  cluster_diameter,
                  cluster_distance, is_admissible, is_leaf, leaf_nodes, EFIECache, build_efie_cache,
                  efie_cache_with_prefactor_scale, aca_lowrank, DenseBlock, LowRankBlock, ACAOperator,
                  ACAAdjointOperator, build_aca_operator)
from ._native import (load_library, LIB_PATH, DiffMoMError, NotConvergedError, FactorizationBreakdown,
                      DeviceWaitTimeout)

__all__ = [n for n in dir() if not n.startswith("_")]
