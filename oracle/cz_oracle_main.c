/* cz-oracle: command-line front end of the CPU restatement (test infrastructure only). Same arguments, stdout
 * format and exit codes as the reference's cheese binary (cheese.cu:1851-1895) for the plain search:
 *   cz-oracle SPEC [--depth D] [--no-dedupe] [--no-sym] [--store64] [--threads T]
 * "seconds" fields are printed as 0.00 (they are machine dependent and never compared). */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "cz_oracle.h"

int main(int argc, char **argv) {
  if (argc < 2) {
    fprintf(stderr, "usage: cz-oracle SPEC [--depth D] [--no-dedupe] [--no-sym] [--store64] [--threads T]\n");
    return 3;
  }
  FILE *f = fopen(argv[1], "rb");
  if (!f) { fprintf(stderr, "not a spec\n"); return 2; }
  fseek(f, 0, SEEK_END);
  const long len = ftell(f);
  fseek(f, 0, SEEK_SET);
  char *text = malloc((size_t)len + 1);
  if (fread(text, 1, (size_t)len, f) != (size_t)len) { fclose(f); return 2; }
  fclose(f);
  text[len] = 0;
  static czo_spec sp;
  char err[256];
  const int prc = czo_spec_parse(text, (size_t)len, &sp, err, sizeof err);
  free(text);
  if (prc) { fprintf(stderr, "%s\n", err); return prc; }
  int depth = sp.depth, dedupe = 1, sym = 1, store64 = 0, threads = 0;
  for (int i = 2; i < argc; i++) {
    if (!strcmp(argv[i], "--depth") && i + 1 < argc) depth = atoi(argv[++i]);
    else if (!strcmp(argv[i], "--no-dedupe")) dedupe = 0;
    else if (!strcmp(argv[i], "--no-sym")) sym = 0;
    else if (!strcmp(argv[i], "--store64")) store64 = 1;
    else if (!strcmp(argv[i], "--threads") && i + 1 < argc) threads = atoi(argv[++i]);
  }
  if (depth > CZO_DMAX) { fprintf(stderr, "depth > %d\n", CZO_DMAX); return 3; }
  static czo_result res;
  const int rc = czo_search(&sp, depth, dedupe, sym, store64, threads, &res);
  fprintf(stderr, "cz-oracle: n %d, %d candidates, depth %d, dedupe %d, %d group elements\n", sp.n, sp.G, depth, dedupe,
          res.nsym);
  if (res.depth0) { printf("{\"found\": 0, \"circuit\": []}\n"); return 0; }
  for (int l = 0; l < res.nlev; l++) {
    const czo_level *v = &res.lev[l];
    printf("{\"t\": %d, \"parents\": %ld, \"prefixes\": %ld, \"cut_w3\": %ld, \"cut_lb\": %ld, \"survivors\": %ld, "
           "\"distinct\": %ld, \"proved_unsat\": %s, \"seconds\": 0.00}\n",
           v->t, v->parents, v->prefixes, v->cut_w3, v->cut_lb, v->survivors, v->distinct,
           v->distinct ? "false" : "true");
  }
  if (rc == 4) { fprintf(stderr, "residual coefficients exceed the storage type: rebuild with -DSTORE64\n"); return 4; }
  if (rc == 0) {
    printf("{\"t\": %d, \"found\": %ld, \"circuit\": [", res.found_len, res.n_found ? res.n_found : 1L);
    for (int i = 0; i < res.found_len; i++) printf("%s\"%s\"", i ? ", " : "", sp.names[res.found[i]]);
    printf("], \"seconds\": 0.00}\n");
  }
  return rc;
}
