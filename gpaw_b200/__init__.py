"""gpaw_b200: GPAW's real-space finite-difference hot path on B200.

Drop-in classes with the reference's Python signatures:

* ``FDOperator``, ``Laplace``, ``GUCLaplace``  (gpaw/fd_operators.py)
* ``Transformer``                               (gpaw/transformers.py)
* ``FDPoissonSolver``                           (gpaw/poisson.py)
* ``Preconditioner``                            (gpaw/preconditioner.py)
* ``GridDescriptor``                            (gpaw/old/grid_descriptor.py)
* ``Gradient``, ``LaplaceA``, ``LaplaceB``      (gpaw/fd_operators.py)
* ``FDHamiltonian``                             (gpaw/new/fd/hamiltonian.py)

and, in their own modules: ``wfd_operators.WeightedFDOperator``
(gpaw/wfd_operators.py), ``solvation.WeightedFDPoissonSolver``
(gpaw/old/solvation/poisson.py), ``dipole.DipoleCorrection``
(gpaw/dipole_correction.py), ``poisson_moment.MomentCorrectionPoissonSolver``
(gpaw/poisson_moment.py), ``poisson_extravacuum.ExtraVacuumPoissonSolver``
(gpaw/poisson_extravacuum.py), ``pot_calc.FDDensityTransfers``
(gpaw/new/fd/pot_calc.py), ``domains`` (the domain decomposition of
gpaw/old/domain.py over a torch.distributed process group); beyond the
reference: ``MixedPoissonSolver``, ``batch.PoissonBatch``, ``serving``,
``pipeline.StepPipeline``, ``autotune`` and ``replicas``.  The C-object
layer is
``gpaw_b200.cgpaw`` (Operator, WOperator, Transformer, fd_precond).  All arrays are torch CUDA tensors; the arithmetic runs in the
sm_100a kernels of ``libgpaw_b200.so`` (C ABI: include/gpaw_b200.h).
"""
from .grid_descriptor import BadGridError, GridDescriptor
from .fd_operators import (FDOperator, Gradient, GUCLaplace, Laplace,
                           LaplaceA, LaplaceB)
from .transformers import Transformer
from .poisson import (FDPoissonSolver, MixedPoissonSolver,
                      PoissonConvergenceError)
from .preconditioner import Preconditioner
from .hamiltonian import FDHamiltonian

__all__ = ['FDHamiltonian', 'Gradient', 'LaplaceA', 'LaplaceB',
           'GridDescriptor', 'BadGridError', 'FDOperator', 'GUCLaplace',
           'Laplace', 'Transformer', 'FDPoissonSolver',
           'MixedPoissonSolver', 'PoissonConvergenceError', 'Preconditioner']
