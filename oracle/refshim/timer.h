/* Stand-in for the CUDA-samples timer header (only main.cu of the reference
 * includes it; that file is not part of the oracle build).  Oracle build recipe only. */
#ifndef GNSS_REFSHIM_TIMER_H
#define GNSS_REFSHIM_TIMER_H
#endif
