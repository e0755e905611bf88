"""CPU oracle of the reference swarm collision path.  TEST INFRASTRUCTURE ONLY: used by tests/,
__graft_entry__.smoke() and bench.py's CPU arms as the checker, never by the product."""
