/* Stand-in for the CUDA-samples header included by the reference; the
 * reference uses nothing from it.  Oracle build recipe only. */
#ifndef GNSS_REFSHIM_HELPER_FUNCTIONS_H
#define GNSS_REFSHIM_HELPER_FUNCTIONS_H
#endif
