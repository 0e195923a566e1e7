/*
 * coinc_io.c -- replacement for the coincidence program's HDF5 I/O
 * (coincidences/io.c) used by the oracle build of coincidences.c (test
 * infrastructure only; libhdf5 is absent from this image).
 *
 *   read_coinc_ini     the reference's own INI reading (io.c:86-154), here
 *                      with the reference's iniparser
 *   read_triggers_file the flat trigger files of oracle/ref_io.c (format 3)
 *                      with the attribute checks of io.c:162-440; the veto
 *                      lines stay zero, as the reference's reader leaves
 *                      them when the search writer has not stored them
 *                      (search io.c:101-106)
 *   init_coin_hdf /
 *   write_coi_hdf      a flat coincidence file under the same name:
 *                        header : char magic[8] = "TDFCOIN1", int32 nseg
 *                        block  : char shift[5], int32 icoi,
 *                                 int32 seginfo[nseg][3],
 *                                 icoi x { int16 w; float avg_snr, avg_f,
 *                                 avg_fdot, avg_ra, avg_dec;
 *                                 int16 cseg[w]; int32 trig_mns[w];
 *                                 int16 n_ccell_trigs[w] }
 *                      one block per shift, in the order they are written
 *   write_ctrigs_hdf   not written (a flag of the reference's that the
 *                      parity runs leave off)
 */
#include <math.h>
#include <stdbool.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "cdefs.h"
#include "../search/network/openmp/struct.h"
#include "coincidences.h"
#include "iniparser.h"

void read_coinc_ini(char *ini_fname, Coinc_opts *copts)
{
     dictionary *ini = iniparser_load(ini_fname);
     if (ini == NULL) {
          perror(ini_fname);
          exit(EXIT_FAILURE);
     }
     copts->refr = iniparser_getint(ini, "coincidences:refr", -1);
     copts->cthr = iniparser_getdouble(ini, "coincidences:cthr", -1.);
     copts->hemi = iniparser_getint(ini, "coincidences:hemi", 1);
     copts->scalef = iniparser_getint(ini, "coincidences:scalef", 1);
     copts->scales = iniparser_getint(ini, "coincidences:scales", 1);
     copts->scalem = iniparser_getint(ini, "coincidences:scalem", 1);
     copts->scalen = iniparser_getint(ini, "coincidences:scalen", 1);
     copts->shift = iniparser_getstring(ini, "coincidences:shift", NULL);
     copts->mincoin = iniparser_getint(ini, "coincidences:mincoin", 4);
     copts->out_dir = iniparser_getstring(ini, "coincidences:out_dir", ".");
     copts->trig_dset = iniparser_getstring(ini, "coincidences:trig_dset", "triggers");
     copts->coinc_dset = iniparser_getstring(ini, "coincidences:coinc_dset", "coinc_");
     copts->write_ctrigs = iniparser_getint(ini, "coincidences:write_ctrigs", 0);
     char *tlist = (char *)iniparser_getstring(ini, "coincidences:trig_file_list", NULL);
     if (copts->refr < 0 || copts->cthr < 0 || !tlist) {
          fprintf(stderr, "Error: invalid or missing parameters in %s\n", ini_fname);
          exit(EXIT_FAILURE);
     }
     size_t count = 0;
     for (char *tok = strtok(tlist, " "); tok != NULL; tok = strtok(NULL, " ")) {
          copts->trig_files[count] = strdup(tok);
          if (++count >= MAX_NSEG) {
               fprintf(stderr, "Error: too many trigger files specified in %s (max %d)\n", ini_fname, MAX_NSEG);
               exit(EXIT_FAILURE);
          }
     }
     copts->nseg = count;
}

static void rd(void *p, size_t sz, size_t n, FILE *f, const char *fn)
{
     if (fread(p, sz, n, f) != n) {
          fprintf(stderr, "Error: short read in %s\n", fn);
          exit(EXIT_FAILURE);
     }
}

size_t read_triggers_file(const char *filename, const char *t_dset_name, Trigger **sgnlv,
                          Search_params *search_par)
{
     (void)t_dset_name;
     const bool init = (search_par->grid_file == NULL);
     FILE *f = fopen(filename, "rb");
     if (!f) {
          fprintf(stderr, "Error: cannot open trigger file %s\n", filename);
          *sgnlv = NULL;
          return 0;
     }
     char magic[8];
     int32_t hdr[2];
     rd(magic, 1, 8, f, filename);
     rd(hdr, sizeof(int32_t), 2, f, filename);
     if (memcmp(magic, "TDFTRIG3", 8) != 0) {
          fprintf(stderr, "Error: %s is not a format-3 trigger file\n", filename);
          exit(EXIT_FAILURE);
     }
     int32_t oi[3];
     double od[2];
     uint32_t gl;
     rd(oi, sizeof(int32_t), 3, f, filename);
     rd(od, sizeof(double), 2, f, filename);
     rd(&gl, sizeof(uint32_t), 1, f, filename);
     char *gf = (char *)calloc(gl + 1, 1);
     rd(gf, 1, gl, f, filename);
     double sd[3];
     int32_t si[5];
     rd(sd, sizeof(double), 3, f, filename);
     rd(si, sizeof(int32_t), 5, f, filename);
     search_par->seg = oi[1];
     if (init) {
          search_par->band = oi[0];
          search_par->hemi = oi[2];
          search_par->overlap = od[0];
          search_par->narrowdown = od[1];
          search_par->grid_file = gf;
          search_par->fpo = sd[0];
          search_par->dt = sd[1];
          search_par->B = sd[2];
          search_par->nod = si[0];
          search_par->N = si[1];
          search_par->nfftf = si[2];
          search_par->numlines_band = si[3];
          search_par->nvlines_all_inband = si[4];
     } else {
          if (search_par->band != oi[0] || search_par->hemi != oi[2] || search_par->overlap != od[0] ||
              search_par->narrowdown != od[1] || strcmp(search_par->grid_file, gf) != 0) {
               fprintf(stderr, "Error: 'opts' attribute in %s does not match expected values\n", filename);
               exit(EXIT_FAILURE);
          }
          if (search_par->nod != si[0] || search_par->N != si[1]) {
               fprintf(stderr, "Error: 'sett' attribute in %s does not match expected values\n", filename);
               exit(EXIT_FAILURE);
          }
          free(gf);
     }
     /* records up to the trailer (len == 0xFFFFFFFF) */
     size_t cap = 1024, n = 0;
     Trigger *t = (Trigger *)malloc(cap * sizeof(Trigger));
     for (;;) {
          float h[6];
          uint32_t len;
          rd(h, sizeof(float), 6, f, filename);
          rd(&len, sizeof(uint32_t), 1, f, filename);
          if (len == 0xFFFFFFFFu) break;
          if (n == cap) {
               cap *= 2;
               t = (Trigger *)realloc(t, cap * sizeof(Trigger));
          }
          t[n].m = h[0];
          t[n].n = h[1];
          t[n].s = h[2];
          t[n].ra = h[3];
          t[n].dec = h[4];
          t[n].fdot = h[5];
          t[n].ffstat.len = len;
          t[n].ffstat.p = len ? malloc(len * sizeof(float)) : NULL;
          if (len) rd(t[n].ffstat.p, sizeof(float), len, f, filename);
          n++;
     }
     fclose(f);
     if (init) search_par->sgnlv_size = n;
     if (n != search_par->sgnlv_size) {
          fprintf(stderr, "Error! sgnlv_size mismatch: read %zu, but expected %zu \n", n, search_par->sgnlv_size);
          exit(EXIT_FAILURE);
     }
     *sgnlv = t;
     return n;
}

int init_coin_hdf(const char *coin_fname, Coinc_opts *copts, Search_params *search_par)
{
     (void)search_par;
     FILE *f = fopen(coin_fname, "wb");
     if (!f) {
          perror(coin_fname);
          exit(EXIT_FAILURE);
     }
     int32_t nseg = (int32_t)copts->nseg;
     fwrite("TDFCOIN1", 1, 8, f);
     fwrite(&nseg, sizeof(int32_t), 1, f);
     fclose(f);
     return 0;
}

int write_coi_hdf(const char *coin_fname, Coinc_opts *copts, Coincidence *coi, int icoi, const char *shift_str,
                  int seginfo[][3])
{
     FILE *f = fopen(coin_fname, "ab");
     if (!f) {
          perror(coin_fname);
          exit(EXIT_FAILURE);
     }
     fwrite(shift_str, 1, 5, f);
     int32_t n = icoi;
     fwrite(&n, sizeof(int32_t), 1, f);
     for (size_t s = 0; s < copts->nseg; s++) {
          int32_t si[3] = {seginfo[s][0], seginfo[s][1], seginfo[s][2]};
          fwrite(si, sizeof(int32_t), 3, f);
     }
     for (int i = 0; i < icoi; i++) {
          const Coincidence *c = &coi[i];
          fwrite(&c->w, sizeof(short), 1, f);
          float v[5] = {c->avg_snr, c->avg_f, c->avg_fdot, c->avg_ra, c->avg_dec};
          fwrite(v, sizeof(float), 5, f);
          fwrite(c->cseg, sizeof(short), c->w, f);
          fwrite(c->trig_mns, sizeof(int), c->w, f);
          fwrite(c->n_ccell_trigs, sizeof(short), c->w, f);
     }
     fclose(f);
     return 0;
}

int write_ctrigs_hdf(const char *ctrigs_fname, Coinc_opts *copts, Search_params *search_par, Coinc_Trigger *ctrigs,
                     int seginfo[][3])
{
     (void)ctrigs_fname; (void)copts; (void)search_par; (void)ctrigs; (void)seginfo;
     return 0;
}
