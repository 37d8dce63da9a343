// Test driver for the reference's own FFT() (FFT.cpp:15-83), used to pin
// the oracle's restatement. TEST INFRASTRUCTURE ONLY.
//   ref_fft <m> <dir>   reads 2^m real then 2^m imaginary doubles on stdin,
//                       writes the transformed arrays the same way on stdout
#include <cstdio>
#include <cstdlib>
#include <vector>

void FFT(short int dir, long m, double x[], double y[]);  // mygeneral.h:126

int main(int argc, char** argv) {
    if (argc != 3) return 2;
    const long m = std::atol(argv[1]);
    const short dir = static_cast<short>(std::atoi(argv[2]));
    const size_t n = size_t(1) << m;
    std::vector<double> x(n), y(n);
    if (std::fread(x.data(), sizeof(double), n, stdin) != n) return 3;
    if (std::fread(y.data(), sizeof(double), n, stdin) != n) return 3;
    FFT(dir, m, x.data(), y.data());
    std::fwrite(x.data(), sizeof(double), n, stdout);
    std::fwrite(y.data(), sizeof(double), n, stdout);
    return 0;
}
