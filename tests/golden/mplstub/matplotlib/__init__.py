"""Import stub: the reference imports matplotlib.path at load time only."""
