"""
macromax_b200: a B200-native (sm_100a) backend for MacroMax's preconditioned modified-Born (split-Richardson)
iteration.  The public API mirrors the reference package: ``solve``, ``Solution``, ``Grid``, the ``bound`` classes
and a ``backend`` module whose ``BackEndB200`` plugs into the reference's ``BackEnd`` registry.
"""
from .grid import Grid
from .bound import Bound, PeriodicBound, AbsorbingBound, LinearBound, Electric, Magnetic
from .solver import Solution, solve

__all__ = ['Grid', 'Bound', 'PeriodicBound', 'AbsorbingBound', 'LinearBound', 'Electric', 'Magnetic',
           'Solution', 'solve']
__version__ = '0.1.0'
