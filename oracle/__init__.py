"""TEST INFRASTRUCTURE ONLY: the checkers (C restatement and the reference
build).  Imported by tests/, __graft_entry__.smoke() and bench.py's CPU legs;
never by the product package."""
from .oracle import ORACLE_SO, REF_SO, Oracle, Reference, build  # noqa: F401
