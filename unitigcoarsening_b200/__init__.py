"""B200-native unitig compactor: hand-written sm_100a CUDA kernels behind the
C ABI of include/uc.h (libuc.so), with a thin Python binding."""
from .api import (CONTRACT_HEC, CONTRACT_POINTER_JUMP, NONE, Compactor, Server, UCError, as_u32, key_words,
                  keys_to_words, lib)

__all__ = ["Compactor", "Server", "UCError", "NONE", "CONTRACT_HEC", "CONTRACT_POINTER_JUMP", "lib", "key_words",
           "keys_to_words", "as_u32"]
