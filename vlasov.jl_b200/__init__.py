"""vlasov_b200: a B200-native (sm_100a) implementation of the per-step
pseudo-particle loop of LaurentPlagne/Vlasov.jl -- stable cell sort, fine and
coarse deposits, nested tensor Poisson solve, smoothed field gather with the
projectile, packed Verlet push -- behind a C ABI (include/vlasov_b200.h).

The directory is named ``vlasov.jl_b200``; it is imported under the module
name ``vlasov_b200`` (see ``load()`` in __graft_entry__.py / tests/conftest.py).
"""
from .tables import (SplineAxis, SplineMesh, NestedMeshes, GaussianSmoothing, LocateTable, uniform_axis,
                     stretched_axis, build_meshes, gaussian_smoothing, smoothing_columns, grids)
from .simulation import (SimulationParameters, Jellium, BallSoftening, GaussianSoftening, Projectile,
                         RadialProfile, read_radial_profile, thomas_fermi_profile, uniform_sphere_profile,
                         sample_thomas_fermi, ran2, pack_positions, unpack_positions, DeviceAccelerator,
                         Simulation, StepDiagnostics, EnergyBudget, Film, xenon_projectile, ThomasFermiStream,
                         STREAM_CHUNK, stream_half_step_cloud, prime_back_chunked)
from . import _lib
from . import xenon
from . import sharded
from . import autotune
from . import sweep
from . import denoiser
from . import precision_run

__all__ = [n for n in dir() if not n.startswith("_")]
