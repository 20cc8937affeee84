/* oco_oracle_run <deck_dir> <out_dir>: runs a reference sample deck through the oracle and
 * writes out_dir/diagnostics.txt (TEST INFRASTRUCTURE ONLY). */
#include <stdio.h>

#include "oco_oracle.h"

int main(int argc, char **argv) {
  if (argc != 3) {
    fprintf(stderr, "usage: %s <deck_dir> <out_dir>\n", argv[0]);
    return 2;
  }
  char msg[512] = "";
  int rc = oracle_run_deck(argv[1], argv[2], msg, sizeof msg);
  if (rc) fprintf(stderr, "oracle: error %d: %s\n", rc, msg);
  return rc ? 1 : 0;
}
