"""B200-native MaoMi optical stage (sm_100a CUDA behind a C ABI)."""

__version__ = "0.1.0"
