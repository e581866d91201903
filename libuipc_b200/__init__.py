"""B200-native Newton-step linear solve (assembly, SpMV, MAS, PCG) with
libuipc's solver/preconditioner interface."""
