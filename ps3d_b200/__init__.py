"""B200-native (sm_100a) engine for the ps3D Boussinesq time step."""
