"""fasterhenry_b200: the PEEC extraction hot path of fasterhenry on B200.

Filament-pair partial-inductance fill, mesh assembly ``Zm = M(R + jwL)M^T``
and a batched complex LU per frequency (FP64, or FP32 with split-BF16 tensor
trailing updates and FP64 iterative refinement), and the matrix-free
precorrected-FFT operator with GMRES, exposed through a C ABI
(include/fasterhenry_b200.h) and this Python mirror of the reference's API.
"""
from .api import (DENSE_PATH_MAX_FILAMENTS, MU0, CoincidentSamples, DiscretizeError, Discretization,
                  FasterHenryError, Geometry, GeometryError, InvalidArgument, InvalidFrequency, InvalidGrading,
                  KernelError, MeshError, MeshSystem, Node, NoDevice, NotConverged, NotFinite, Port, Precision,
                  SegmentDef, Singular, SolverChoice, SweepResult, Unsupported, build_info, device_count, discretize,
                  lu_solve, mesh_matrix, mutual_inductance, partial_inductance_matrix, self_inductance, skin_depth,
                  solve)
from .api import (GmresOutcome, GmresParams, IterativeParams, IterativeSystem, PfftError, PfftOperator, PfftParams,
                  Profiler, batch_sweep, fill_stats, gmres_dense)
from .api import (GradientResult, Param, coordinate_gradient, grid_convolution, inductance_gradient, near_pairs,
                  release_cached_memory)
from .api import CURRENTS_CSV_HEADER, CurrentSolution, InvalidExcitation, unit_excitation
from .api import DEFAULT_GROUP, Coupling, CouplingError, TruncationWarning
from . import problem
from .problem import DeckError, DeckWarning, Problem, ProblemError, load, parse_deck, parse_deck_reporting, run

__version__ = "0.1.0"
