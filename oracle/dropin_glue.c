/*
 * dropin_glue.c -- links the reference's search() host to libtdfcuda
 * (integration test build, oracle/Makefile target `dropin`).  The reference's
 * jobcore.c is compiled unmodified and its job_core() made a weak symbol
 * (objcopy --weaken-symbol); this strong definition, with the reference's
 * signature (search/network/openmp/jobcore.h:21-33), takes its place and
 * forwards to the library's drop-in entry tdf_job_core_ref().  A maintainer
 * who can edit jobcore.c instead removes its job_core() and links
 * libtdfcuda directly (the library also exports job_core()).
 */
#include "tdfcuda_refabi.h"

int job_core(int pm, float mm, float nn, tdf_ref_Search_settings *sett, tdf_ref_Command_line_opts *opts,
             tdf_ref_Search_range *s_range, void *plans, void *fftw_arr, tdf_ref_Aux_arrays *aux,
             int *sgnlc, tdf_ref_Trigger *sgnlv, int *FNum)
{
     return tdf_job_core_ref(pm, mm, nn, sett, opts, s_range, plans, fftw_arr, aux, sgnlc, sgnlv, FNum);
}
