"""blastp_b200: host layer of the B200 blastp preliminary-search engine.

The engine (two-hit word finding + BLOSUM62 X-drop ungapped extension) is the
CUDA library libblastp_b200.so; this package binds its C ABI and provides the
synthetic-data generators used by the benchmark and the tests.
"""
from . import synth  # noqa: F401
from ._lib import BpError, BpParams, lib  # noqa: F401
from .api import (GAPPED_DTYPE, HSP_DTYPE, Batch, Database, Engine, GappedResult, Mlp, PendingResult,  # noqa: F401
                  Query, Result, Server, blosum62, default_params, gapped_params, read_database_file,
                  write_database_file)
from . import costmodel  # noqa: F401,E402
