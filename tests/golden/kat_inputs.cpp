// kat_inputs.cpp -- regenerates the exact seeded inputs of the reference's
// own tests (they hold no stored vectors; they draw from std::mt19937 /
// std::mt19937_64 and std::normal_distribution at run time).  Built and run
// by make_golden.py; output is raw float32 arrays, one file per case.
//
// Draw orders follow the reference tests:
//   tests/cffi_stft_compare_test.cpp:237-242  fill_random (normal<float>)
//   tests/fftfree_tests.cpp:176-190           roundtrip (mt19937_64, re then im)
//   tests/fftfree_tests.cpp:275-285           reference_batch (row-major, re[, im])
//   tests/fftfree_tests.cpp:422-433           prepared transform (mt19937)
//   tests/fftfree_tests.cpp:1277-1304         multi-N metadata (mt19937_64, shared)
#include <cstdio>
#include <complex>
#include <cstdint>
#include <cstdlib>
#include <random>
#include <string>
#include <vector>

static void dump(const std::string& dir, const std::string& name, const std::vector<float>& v) {
  const std::string path = dir + "/" + name + ".f32";
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) { std::perror(path.c_str()); std::exit(1); }
  std::fwrite(v.data(), sizeof(float), v.size(), f);
  std::fclose(f);
}

// N x frames complex matrix, drawn row by row (r over N, c over frames),
// stored here as interleaved complex in that same row-major (r, c) order.
static std::vector<float> reference_batch(int N, int frames, unsigned seed, bool complex_kind) {
  std::vector<float> out(static_cast<size_t>(N) * frames * 2, 0.0f);
  std::mt19937 rng(seed);
  std::normal_distribution<double> dist(0.0, 1.0);
  for (int r = 0; r < N; ++r) {
    for (int c = 0; c < frames; ++c) {
      const float re = static_cast<float>(dist(rng));
      const float im = complex_kind ? static_cast<float>(dist(rng)) : 0.0f;
      out[(static_cast<size_t>(r) * frames + c) * 2] = re;
      out[(static_cast<size_t>(r) * frames + c) * 2 + 1] = im;
    }
  }
  return out;
}

int main(int argc, char** argv) {
  if (argc < 2) { std::fprintf(stderr, "usage: kat_inputs <outdir>\n"); return 2; }
  const std::string dir = argv[1];

  {  // plain FFT via the C ABI, N=1024, mt19937(1337)
    std::vector<float> pcm(1024);
    std::mt19937 rng(1337);
    std::normal_distribution<float> dist(0.0f, 1.0f);
    for (float& s : pcm) s = dist(rng);
    dump(dir, "cffi_plain_fft_pcm", pcm);
  }
  {  // batched STFT via the C ABI, N=W=512, H=128, 8 frames, mt19937(42)
    std::vector<float> pcm(512 + 7 * 128);
    std::mt19937 rng(42);
    std::normal_distribution<float> dist(0.0f, 1.0f);
    for (float& s : pcm) s = dist(rng);
    dump(dir, "cffi_batched_stft_pcm", pcm);
  }
  {  // roundtrip N=16, B=8, mt19937_64(42), signal(i, j) re then im
    const int N = 16, B = 8;
    std::vector<float> x(static_cast<size_t>(N) * B * 2);
    std::mt19937_64 rng(42);
    std::normal_distribution<double> dist(0.0, 1.0);
    for (int i = 0; i < N; ++i)
      for (int j = 0; j < B; ++j) {
        x[(static_cast<size_t>(i) * B + j) * 2] = static_cast<float>(dist(rng));
        x[(static_cast<size_t>(i) * B + j) * 2 + 1] = static_cast<float>(dist(rng));
      }
    dump(dir, "roundtrip_n16_b8", x);
  }
  dump(dir, "single_thread_n8_b3_s1381", reference_batch(8, 3, 1381u, true));
  {  // prepared transform N=64, B=4, mt19937(1337)
    const int N = 64, B = 4;
    std::vector<float> x(static_cast<size_t>(N) * B * 2);
    std::mt19937 rng(1337);
    std::normal_distribution<double> dist(0.0, 1.0);
    for (int r = 0; r < N; ++r)
      for (int c = 0; c < B; ++c) {
        x[(static_cast<size_t>(r) * B + c) * 2] = static_cast<float>(dist(rng));
        x[(static_cast<size_t>(r) * B + c) * 2 + 1] = static_cast<float>(dist(rng));
      }
    dump(dir, "prepared_n64_b4", x);
  }
  dump(dir, "stockham_n256_b128_s1337", reference_batch(256, 128, 1337u, false));
  dump(dir, "stockham_n256_b128_s2337", reference_batch(256, 128, 2337u, false));
  dump(dir, "twiddle_meta_n16_b5_s2025", reference_batch(16, 5, 2025u, true));
  dump(dir, "consensus_n8_b3_s2026", reference_batch(8, 3, 2026u, true));
  for (int N : {2, 4, 8, 16, 32}) {
    for (int frames : {1, 3, 16}) {
      const unsigned seed = static_cast<unsigned>(N * 1009 + frames * 97);
      dump(dir, "extended_n" + std::to_string(N) + "_b" + std::to_string(frames),
           reference_batch(N, frames, seed, true));
    }
  }
  {  // multi-N metadata: one mt19937_64(123456) shared across N = 1,2,4,8,16
    std::mt19937_64 rng(123456);
    std::normal_distribution<double> dist(0.0, 1.0);
    for (int N : {1, 2, 4, 8, 16}) {
      const int frames = 3;
      std::vector<float> x(static_cast<size_t>(N) * frames * 2);
      // The reference draws both parts inside one constructor call, whose
      // argument evaluation order is the compiler's; the same expression
      // form is used here so the same compiler picks the same order.
      for (int r = 0; r < N; ++r)
        for (int c = 0; c < frames; ++c) {
          const std::complex<float> v = std::complex<float>(static_cast<float>(dist(rng)),
                                                            static_cast<float>(dist(rng)));
          x[(static_cast<size_t>(r) * frames + c) * 2] = v.real();
          x[(static_cast<size_t>(r) * frames + c) * 2 + 1] = v.imag();
        }
      dump(dir, "multin_meta_n" + std::to_string(N), x);
    }
  }
  return 0;
}
