"""CPU oracle for the ERTM RTM hot path.

TEST INFRASTRUCTURE ONLY.  Nothing in the product package imports this
directory.  Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s
CPU-baseline / reference arm may import it, and only as the checker.

The oracle is a NumPy restatement of the reference algorithm
(Sherlyn7189/Challenge-Cup, ``ertm/numerics.py``, ``ertm/propagation.py``,
``ertm/imaging.py``, ``ertm/viscoelastic.py``, ``ertm/pipeline.py``).  It is
pinned against golden vectors produced by running the reference itself
(``tests/golden/make_golden.py`` → ``tests/golden/*.npz``); the CPU test
suite checks it against every one of them.
"""

from .ertm_oracle import *  # noqa: F401,F403
