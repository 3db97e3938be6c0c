"""CPU checkers for the LOITS sampler (test infrastructure, never the product).

``oracle.oracle`` wraps the plain-C restatement (``loits_oracle.c``) and the
reference's own compiled cores (``_ref/``).  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline / reference arm
import this package; ``quantom_loits_b200`` never does.
"""
