"""frforge_b200: B200-native FP64 FR residual + SSP-RK time-step path.

Drop-in for FRForge's hot path (src/fr, src/flux, src/capturing, src/time,
src/solvestate): the residual, the capturing hooks and the SSP-RK loop run in
``libfrforge_cuda.so`` (sm_100a kernels) behind the C ABI in
``include/frforge_cuda.h``.  This package is the host-side mirror of the
reference's Julia API.
"""
from .equations import Euler1D, Euler2D
from .gpu import (Context, GpuSolve, compute_dt, default_context, integrate_, residual_, sense_,
                  ssp_rk2_, ssp_rk2_step_, ssp_rk3_, ssp_rk3_step_)
from .mesh import (DirichletBC, Mesh1D, Mesh2D, PeriodicBC, ReflectingBC, TransmissiveBC,
                   XSplitGhostBC, is_periodic, julia_range, make_wavy_mesh2d)
from .methods import (AbstractCapturingMethod, ElementArtificialViscosity, NullCapturing,
                      PerssonAVMethod, PerssonSensor, PositivityPreservingPersson, ScaledPerssonMethod, FluxOverridePersson,
                      PositivityPreprocessPersson, TraceOverridePersson,
                      get_capturing_method, list_methods, method_params, register_method)
from .operators import FROperators, build_operators, n_points
from .scheme import DEFAULT_SCHEME, SchemeConfig, parse_scheme, scheme_dict
from .state import (SolutionState, SolutionState2D, allocate_state, discrete_mass, has_nonfinite,
                    positivity_ok, set_initial_condition_, solution_extrema)
from .vtk import (VTK_LAGRANGE_LINE, VTK_LAGRANGE_QUAD, write_vtu_high_order,
                  write_vtu_high_order_with_capturing)
from ._lib import FRGError, UnsupportedHookError

__all__ = [n for n in dir() if not n.startswith("_")]
