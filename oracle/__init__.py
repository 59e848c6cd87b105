"""CPU oracle for the Simulon per-step force path.

TEST INFRASTRUCTURE ONLY.  Nothing in the ``simulon_b200`` product package
imports, links or calls this package.  Only ``tests/``, ``__graft_entry__.smoke()``
and the CPU-baseline legs of ``bench.py`` use it, and only as the checker or
as the timed CPU baseline -- never as a substitute for the CUDA path.

The oracle restates the reference algorithms (JinZongxiao/Simulon) on the CPU:

* ``box``        -- minimum image / wrap            (core/box.py:109-142)
* ``neighbor``   -- half Verlet list i<j            (core/neighbor_search/gpu_kdtree.py:90-155,
                                                     io_utils/reader.py:364-376,477-484)
                    implemented in C (``neighbor_ref.c``) with the exact op order
                    that torch's CPU kernels use, so the pair set is bit-exact.
* ``lj``         -- Lennard-Jones forward           (core/force/lennard_jones_force.py:15-95)
* ``eam``        -- setfl/FS parser, uniform tables, two-pass forward
                    (io_utils/eam_parser.py:23-210, core/force/eam_force_cu.py:334-579)
* ``integrator`` -- velocity Verlet / Langevin / Berendsen / BaseModel order
                    (core/integrator/integrator.py:45-124, core/barostat.py:36-68,
                     core/md_model.py:88-166)
* ``philox``     -- Philox4x32-10 + Box-Muller, the counter-based noise the
                    CUDA Langevin kernel also uses (so noise can be reproduced)
* ``inputs``     -- seeded synthetic systems (FCC Ar, BCC W, triclinic, FS-W setfl file)

Parity is pinned against golden vectors produced by running the reference
itself (``tests/golden/make_golden.py``); see ``tests/test_oracle_golden.py``.
"""
