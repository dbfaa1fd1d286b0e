"""Drop-in, B200-native DEM droplet hot path (see the package README in DESIGN.md)."""
