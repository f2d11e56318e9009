"""CPU oracle of the propagator and Parareal driver (test infrastructure only)."""
