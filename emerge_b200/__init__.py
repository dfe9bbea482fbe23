"""B200-native Nedelec-2 curl-curl assembly for EMerge (drop-in for the
``tet_mass_stiffness_matrices`` / ``CSCMapping.to_csc`` hot path)."""
__version__ = "0.1.0"
