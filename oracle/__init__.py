"""CPU oracle for the dynamics_b200 nonbonded/MD engine.

TEST INFRASTRUCTURE ONLY.  Nothing in the product package imports this
package; only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline
legs of ``bench.py`` use it, and only as the checker or as the timed CPU
restatement of the reference path.

The reference (David-OConnor/dynamics, Rust crate ``dynamics`` 0.2.2) cannot
be compiled in this environment (no Rust toolchain, crates not vendored), so
every function here is a restatement of the reference's algorithm, citing the
reference file:line it follows:

* ``opc``        -- OPC rigid-water constants and geometry
                    (src/solvent/mod.rs, src/solvent/opc_settle.rs)
* ``pairs``      -- neighbour lists, flat pair assembly and the short-range
                    LJ + erfc Coulomb pair math (src/neighbors.rs,
                    src/non_bonded.rs, src/cuda/cuda.cu, src/barostat.rs)
* ``spme``       -- smooth PME (Essmann et al. 1995, order-4 cardinal
                    B-splines).  The reference calls the external crate
                    ``ewald`` ^0.1.15 (Cargo.toml:42), whose source is not in
                    the reference tree; this is a restatement of the published
                    method at the reference's call sites
                    (src/non_bonded.rs:681-875) and is pinned by the
                    reference's own physical tests (src/tests/spme.rs) plus a
                    direct Ewald sum.
* ``integrate``  -- rigid water drift, kicks, Langevin OU, CSVR, KE/pressure
                    (src/integrate.rs, src/thermostat.rs, src/barostat.rs)
* ``philox``     -- Philox4x32-10 counter RNG (Salmon et al., SC'11), the
                    same stream the CUDA engine draws, so stochastic steps
                    are comparable.
* ``bonded``     -- bonds, angles, dihedrals, H constraints
                    (src/bonded.rs, src/bonded_forces.rs)
* ``cpu_ref/``   -- C++17/OpenMP restatement of the reference CPU step
                    (O(N^2) Verlet build, flat pair list, per-thread f64
                    accumulation, SPME with a CPU FFT, serial rigid water),
                    used as the timed CPU baseline.

Parity status: the reference ships no golden vectors or fixtures.  The
restatement is pinned against the reference's inline known-answer tests
(src/tests/forces.rs, src/tests/spme.rs, src/tests/force_components.rs,
src/tests/therm_baro.rs), re-expressed in tests/test_oracle_*.py.  Bitwise
SPME parity with the ``ewald`` crate is unpinned (its source is absent).
"""
