"""CPU oracle of the graph-index build path: test infrastructure only."""
