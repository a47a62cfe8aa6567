"""classicaldft_b200: the classicalDFT F[rho] / dF/drho hot path on NVIDIA B200.

The compute path is libcdft_b200.so (hand-written sm_100a CUDA kernels, cuFFT
for the batched R2C/C2R plans) behind the C ABI of include/cdft_b200.h.
This package is the Python host API over that ABI, mirroring the reference
library's functional interface.
"""
from ._lib import FP64, MIXED, EngineError, lib  # noqa: F401
from .functionals import (BARKER_HENDERSON, WEEKS_CHANDLER_ANDERSEN, Engine, EsFMT, FMTModel, Functional,  # noqa: F401
                          Grid, Interaction, Model, Potential, Result, Rosenfeld, RSLT, Species, Weights,
                          WhiteBearI, WhiteBearII, interaction_weight, make_grid, make_lennard_jones,
                          make_ten_wolde_frenkel, make_wang_ramirez_dobnikar_frenkel, make_weights, total,
                          total_batch, total_stream)

from .algorithms import set_step_graphs, step_graphs  # noqa: F401
from .algorithms import (Bounded, EigenvalueResult, EigenvalueSolver, Fire, FixedMassConstraint,  # noqa: F401
                         MinimizationResult, Minimizer, Picard, PicardResult, ReservoirBoundary, SaddleResult, Search,
                         Simulation, Snapshot, StepConfig, Unbounded, crank_nicholson_step, fixed_mass_constraint,
                         ddft_last_step, hessian_times_vector, integrating_factor_step, reservoir_boundary,
                         split_operator_step)
from .bulk import (BulkThermodynamics, Coexistence, PhaseSearch, Spinodal, density_from_chemical_potential,  # noqa: F401
                   densities_from_chemical_potentials, make_bulk_thermodynamics, make_bulk_weights)

__version__ = "0.1.0"
