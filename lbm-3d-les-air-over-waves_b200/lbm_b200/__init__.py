"""B200-native D3Q19 step engine for the air-over-waves LES / free-surface
solver (drop-in for the per-timestep path of
LBM_3D_LES_air_over_waves_CODEX.py)."""
