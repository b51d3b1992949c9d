"""uaamg_b200: B200-native UAAMG-PCG (pressure Poisson + variational viscosity)."""
