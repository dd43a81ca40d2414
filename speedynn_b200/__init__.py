"""B200-native greedy nearest-neighbour wrapper feature selection."""
__version__ = "0.1.0"
