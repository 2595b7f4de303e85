"""B200-native 3D time-domain EM edge-FEM forward solve (grounded-wire source)."""
