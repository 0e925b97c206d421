"""B200 (sm_100a) channel-flow hot path: the x-z transforms, dealiased
nonlinear products and per-wavenumber implicit y-solves of the reference
Fortran solver, behind the C ABI of include/chanflow.h."""
from .chanflow import (FP64, MIXED, CfgFringe, CfgJet, CfgLes, ChanflowError, ChannelFlow, Ensemble, Grid, Group, Mlp,  # noqa: F401
                       Rank,
                       initial_field, load_library, partition, read_flow_dat, read_velocity_file,
                       save_velocity_file, LIB_PATH, PARTITION_KEYS, SYMBOLS)
