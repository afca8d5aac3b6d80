"""hydra_lotus_b200: a B200-native (sm_100a) CUDA backend for hydra-lotus's
integrator hot path, behind the reference's OffscreenRenderer contract."""
