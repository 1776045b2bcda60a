"""CPU oracle for PHEM's CC/SF and MSF hot paths.

TEST INFRASTRUCTURE ONLY: the parity tests, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` use it as the checker.  The product package
``phem_graph_b200`` never imports it.
"""
from .oracle import *  # noqa: F401,F403
