"""CPU oracle for the diffmpc inner QP solve (test infrastructure only).

This package restates, in torch float64 on the CPU, the algorithm of the
reference solver (ToyotaResearchInstitute/diffmpc):

* ``models``      -- ``state_dot`` of the linear, quadrotor, spacecraft-rate,
                     spacecraft-attitude and cart-pole models
                     (``diffmpc/dynamics/*_dynamics.py``);
* ``integrators`` -- ``predict_next_state`` (``diffmpc/dynamics/integrators.py:20-71``);
* ``ocp``         -- ``OptimalControlProblem`` (``diffmpc/problems/optimal_control_problem.py``);
* ``pcg``         -- ``PCGOptimalControl`` (``diffmpc/solvers/pcg.py``);
* ``sqp``         -- ``SQPSolver`` forward, line search and the implicit-function
                     backward (``diffmpc/solvers/sqp.py``).

It is the checker, never the product: only ``tests/``, ``__graft_entry__.smoke()``
and ``bench.py``'s CPU-baseline / reference arm may import it.  The product
path (``diffmpc_b200``) never routes through this package.

Parity pins: the oracle is checked against the reference's own recorded
outputs (the RL notebooks' losses and post-step weights, the imitation
learning demonstrations) and the assertions of the reference's tests; see
``tests/test_oracle_pins.py``.

Batching follows ``jax.vmap`` of ``lax.while_loop``: every tensor carries a
leading batch dimension, loops run while any lane is active and finished
lanes are frozen with a select, so per-lane results equal unbatched ones.
All arithmetic is float64 (the reference sets ``jax_enable_x64``).
"""

F64 = "float64"
