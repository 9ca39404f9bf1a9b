"""Oracle for the path-tracing core: TEST INFRASTRUCTURE ONLY.

Two checkers live here:
  _ref/liboracle_ref.so  the reference renderer's own C++ sources compiled with
                         project-written glm/spdlog/stb shims and a harness
                         (Makefile, shim/, harness/); wrapped by oracle.ref.
  _ref/liboracle_port.so a plain-C restatement of the reference's traversal and
                         path integrator (restate/); wrapped by oracle.port.
Only tests, __graft_entry__.smoke() and bench.py's CPU-baseline leg load them,
and only to check or time the reference; the product never calls into them.
"""
