"""Debug verbosity thresholds, compared with `debug_verb` (paces/config/dbg_verbosity_levels.py:19-48).

A message is printed when debug_verb exceeds its level; raise a level to silence it.
"""

# initialisation messages (printed once at the start of a calculation)
INIT_VERBOSITY_LEVEL = 0
# per-step checkpoints (new Hilbert space, propagation, observables)
BASE_STEP_LEVEL = 1
# details of each evolution of the Hilbert space
HILBERT_SPACE_LEVEL = 2
# even more details of each evolution of the Hilbert space
HILBERT_SPACE_DETAILED_LEVEL = 4
# status of individual observables
OBSERVABLES_LEVEL = 3
# norm at every term of the series expansion of U(dt)
EXPM_EVO_LEVEL = 6
# memory use
MEM_INFO_LEVEL = 5
# inter-device transfer times
MOVE_DATA_TIMING_LEVEL = 5
# lookup timings
SEARCHSORTED_TIMING_LEVEL = 7
