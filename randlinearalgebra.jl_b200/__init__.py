"""B200-native RandLinearAlgebra.jl sketch / RandSVD path: the host-side mirror of the
reference's Compressor and RangeApproximator API over librla_b200.so.

The directory name is not a Python identifier; load it with
``__graft_entry__.load_package()`` (module name ``randlinearalgebra_b200``).
"""
from .errors import ArgumentError, DimensionMismatch, DomainError, RLAError
from .compressors import (Cardinality, Left, Right, Undef, Compressor, CompressorRecipe, CompressorAdjoint,
                          SparseSign, SparseSignRecipe, CountSketch, CountSketchRecipe, SRHT, SRHTRecipe, FJLT,
                          FJLTRecipe, Gaussian, GaussianRecipe, complete_compressor, update_compressor_, mul_,
                          adjoint, transpose, size, seed_)
from .approximators import (Approximator, RangeApproximator, ApproximatorRecipe, RangeApproximatorRecipe,
                            ApproximatorAdjoint, RangeFinder, RangeFinderRecipe, RandSVD, RandSVDRecipe,
                            complete_approximator, rapproximate_, rapproximate, RandSVDBatch)
from ._lib import RLA_PREC_NATIVE, RLA_PREC_SPLIT_BF16, lib, Context
from .serving import Server, sketch_solve
from .sampling import (Sampling, SamplingRecipe, Distribution, DistributionRecipe, Uniform, UniformRecipe, L2Norm,
                       L2NormRecipe, Agmon, AgmonRecipe, complete_distribution, update_distribution_,
                       sample_distribution_)
from .solvers import (Solver, SolverRecipe, Logger, LoggerRecipe, SolverError, SolverErrorRecipe, BasicLogger,
                      BasicLoggerRecipe, threshold_stop, complete_logger, update_logger_, reset_logger_, FullResidual,
                      FullResidualRecipe, LSGradient, LSGradientRecipe, CompressedResidual, CompressedResidualRecipe,
                      complete_error, compute_error, IHS, IHSRecipe, complete_solver, rsolve_, SubSolver,
                      SubSolverRecipe, LQSolver, LQSolverRecipe, QRSolver, QRSolverRecipe, complete_sub_solver,
                      update_sub_solver_, ldiv_, Kaczmarz, KaczmarzRecipe, ColumnProjection, ColumnProjectionRecipe)

__version__ = "0.1.0"
