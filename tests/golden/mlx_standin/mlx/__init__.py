"""Empty package: the stand-in for mlx (see core.py)."""
