"""vxr: the B200-native rigid-body step behind a C-ABI (``include/vxr.h``), and its host-side mirror of the
reference's simulation API (BoxSimulation / SphereSimulation of sibarum/vexelray-sim-rigid)."""
