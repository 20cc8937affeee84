/*
 * flux_feautrier_b200 -- command-line counterpart of the reference's executable
 * (./source/flux_feautrier.x [snapshot], flux_feautrier.f90:63-66), run in a deck directory
 * (input.in, resolution.in, input_athena/); writes output/ as the reference does, with the
 * xy/lambda loop on the GPU.
 *
 *   flux_feautrier_b200 [snapshot] [--form plain|stable|mixed] [--device N] [--no-binary]
 *                       [--deck DIR] [--out DIR]
 */
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "oco.h"

int main(int argc, char **argv) {
  std::string snapshot = "0000", deck = ".", out;
  int form = OCO_FORM_PLAIN, device = 0, binary = 1;
  for (int i = 1; i < argc; i++) {
    const std::string a = argv[i];
    if (a == "--form" && i + 1 < argc) {
      const std::string f = argv[++i];
      form = f == "plain" ? OCO_FORM_PLAIN : f == "stable" ? OCO_FORM_STABLE : f == "mixed" ? OCO_FORM_MIXED : -1;
      if (form < 0) {
        fprintf(stderr, "unknown form %s\n", f.c_str());
        return 2;
      }
    } else if (a == "--device" && i + 1 < argc) {
      device = atoi(argv[++i]);
    } else if (a == "--deck" && i + 1 < argc) {
      deck = argv[++i];
    } else if (a == "--out" && i + 1 < argc) {
      out = argv[++i];
    } else if (a == "--no-binary") {
      binary = 0;
    } else if (!a.empty() && a[0] != '-') {
      snapshot = a;
    } else {
      fprintf(stderr, "usage: %s [snapshot] [--form plain|stable|mixed] [--device N] [--no-binary] "
                      "[--deck DIR] [--out DIR]\n", argv[0]);
      return 2;
    }
  }
  oco_deck_info info{};
  if (oco_deck_block_inputs(deck.c_str(), snapshot.c_str(), 0, 0, &info, nullptr, nullptr, nullptr, nullptr)) {
    fprintf(stderr, "%s\n", oco_deck_last_error());
    return 1;
  }
  if (info.lread_athena) printf(" snapshot: %s\n", snapshot.c_str());
  const auto t0 = std::chrono::steady_clock::now();
  const int rc = oco_run_deck(deck.c_str(), snapshot.c_str(), out.c_str(), form, device, binary);
  const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (rc) {
    fprintf(stderr, "%s\n", oco_deck_last_error());
    if (rc != OCO_EZEROPIVOT) return 1;
  }
  const double pts = (double)info.nz * info.ny * info.nx * info.nw;
  printf("\n Wall time = %g seconds.\n", s);
  printf(" Execution time = %g micro-seconds per wavelength point per mesh point.\n", s / pts * 1e6);
  return rc ? 1 : 0;
}
