/*
 * ref_io.c -- replacement for the reference's HDF5 trigger writer
 * (search/network/openmp/io.c:16-281) used by the oracle builds (test
 * infrastructure only).  libhdf5 is absent from this image, so the same
 * records are written to a flat little-endian file under the same name:
 *
 *   header : char magic[8] = "TDFTRIG3", int32 format_version (=3), int32 nifo,
 *            then the attributes the reference writes (io.c:44-105) that a
 *            trigger consumer reads (coincidences/io.c:197-300):
 *              opts: int32 band, seg, hemi; double overlap, narrowdown;
 *                    uint32 n + n bytes grid_file
 *              sett: double fpo, dt, B; int32 nod, N, nfftf, numlines_band,
 *                    nvlines_all_inband
 *            (the veto lines themselves are not an attribute: the
 *            reference's writer leaves them out, io.c:101-106)
 *   record : float m, n, s, ra, dec, fdot;  uint32 len;  float ffstat[len]
 *            (the Trigger compound of io.c:34-42 / struct.h:211-215; len
 *            counts floats, two per trigger: f then F)
 *   trailer: six NaN floats, uint32 0xFFFFFFFF, int32 totsgnl,
 *            double walltime, int32 num_threads (io.c:272-276 attributes)
 *
 * hdfout_init truncates the file as H5Fcreate(H5F_ACC_TRUNC) does (io.c:138).
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "auxi.h"
#include "struct.h"

#define REFIO_FORMAT_VERSION 3

int hdfout_init(char *outname, Command_line_opts *opts, Search_settings *sett,
                Search_range *s_range, Trigger *sgnlv)
{
     (void)s_range; (void)sgnlv;
     FILE *f = fopen(outname, "wb");
     if (!f) { perror(outname); exit(EXIT_FAILURE); }
     const char magic[8] = {'T', 'D', 'F', 'T', 'R', 'I', 'G', '3'};
     int32_t hdr[2] = {REFIO_FORMAT_VERSION, sett->nifo};
     fwrite(magic, 1, 8, f);
     fwrite(hdr, sizeof(int32_t), 2, f);
     int32_t oi[3] = {opts->band, opts->seg, opts->hemi};
     double od[2] = {opts->overlap, opts->narrowdown};
     const char *gf = opts->grid_file ? opts->grid_file : "";
     uint32_t gl = (uint32_t)strlen(gf);
     fwrite(oi, sizeof(int32_t), 3, f);
     fwrite(od, sizeof(double), 2, f);
     fwrite(&gl, sizeof(uint32_t), 1, f);
     fwrite(gf, 1, gl, f);
     double sd[3] = {sett->fpo, sett->dt, sett->B};
     int32_t si[5] = {sett->nod, sett->N, sett->nfftf, sett->numlines_band, sett->nvlines_all_inband};
     fwrite(sd, sizeof(double), 3, f);
     fwrite(si, sizeof(int32_t), 5, f);
     fclose(f);
     return EXIT_SUCCESS;
}

int hdfout_extend(char *outname, Trigger *sgnlv, int sgnlv_size)
{
     FILE *f = fopen(outname, "ab");
     if (!f) { perror(outname); exit(EXIT_FAILURE); }
     for (int r = 0; r < sgnlv_size; r++) {
          float hdr[6] = {sgnlv[r].m, sgnlv[r].n, sgnlv[r].s,
                          sgnlv[r].ra, sgnlv[r].dec, sgnlv[r].fdot};
          uint32_t len = (uint32_t)sgnlv[r].ffstat.len;
          fwrite(hdr, sizeof(float), 6, f);
          fwrite(&len, sizeof(uint32_t), 1, f);
          if (len) fwrite(sgnlv[r].ffstat.p, sizeof(float), len, f);
     }
     fclose(f);
     return EXIT_SUCCESS;
}

int hdfout_finalize(char *outname, int totsgnl, double time_elapsed, int nthreads)
{
     FILE *f = fopen(outname, "ab");
     if (!f) { perror(outname); exit(EXIT_FAILURE); }
     float nanv[6];
     for (int i = 0; i < 6; i++) nanv[i] = NAN;
     uint32_t end = 0xFFFFFFFFu;
     int32_t ts = totsgnl, nt = nthreads;
     fwrite(nanv, sizeof(float), 6, f);
     fwrite(&end, sizeof(uint32_t), 1, f);
     fwrite(&ts, sizeof(int32_t), 1, f);
     fwrite(&time_elapsed, sizeof(double), 1, f);
     fwrite(&nt, sizeof(int32_t), 1, f);
     fclose(f);
     return EXIT_SUCCESS;
}
