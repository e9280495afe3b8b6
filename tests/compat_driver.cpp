// compat_driver.cpp -- test driver for the drop-in FREESTREAMMILNE class: reads
// the initial energy density (GeV/fm^3, float32 binary) from argv[1], runs the
// class in the current directory (freestream_input, output/), and writes the
// 17 output vectors (float64 binary, reference order) and tau_LandauMatch to
// argv[2].  Mirrors how src/RunWrapper.cpp drives the reference class.
#include <cstdio>
#include <vector>

#include "FreestreamMilne.cpp"

int main(int argc, char** argv) {
  if (argc != 3) return 2;
  std::vector<float> e;
  FILE* f = fopen(argv[1], "rb");
  if (!f) return 3;
  float v;
  while (fread(&v, 4, 1, f) == 1) e.push_back(v);
  fclose(f);
  FREESTREAMMILNE fs;
  fs.initialize_from_vector(e);
  int rc = fs.run_freestream_milne();
  std::vector<double> o[17];
  fs.output_to_vectors(o[0], o[1], o[2], o[3], o[4], o[5], o[6], o[7], o[8], o[9], o[10], o[11],
                       o[12], o[13], o[14], o[15], o[16]);
  FILE* g = fopen(argv[2], "wb");
  if (!g) return 4;
  double tau = fs.tau_LandauMatch;
  fwrite(&tau, 8, 1, g);
  for (auto& x : o) fwrite(x.data(), 8, x.size(), g);
  fclose(g);
  return rc;
}
