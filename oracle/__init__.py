"""CPU oracle of the HSGeneral stochastic path -- test infrastructure only."""
