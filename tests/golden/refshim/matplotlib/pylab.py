"""Empty stand-in for matplotlib.pylab."""
