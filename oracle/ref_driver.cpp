// Trace driver for the reference interpreter (CPU oracle and CPU baseline).
//
// Each subcommand records one chai trace through the reference's public API
// (api/chai.h) and reads the result back, so the trace runs on the reference's
// bytecode interpreter device (runtime/Interpreter.cpp:335-363).  Inputs come
// from raw little-endian files through make1/make2 (api/ArrayFP.cpp:247-357),
// because the interpreter's own RNG is glibc random_r salted with an object
// address and cannot be reproduced (interp/InterpRNG.cpp:18-22).
//
// Output: result arrays as raw files, and one line on stdout
//   "ms=<wall milliseconds of the traced section> <name>=<value> ..."
//
// Test infrastructure only; the product never links or runs this program.

#include <chai/chai.h>

#include <sys/time.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <sstream>
#include <string>
#include <vector>

using namespace chai;
using namespace std;

static double now_ms()
{
    struct timeval tv;
    gettimeofday(&tv, 0);
    return tv.tv_sec * 1e3 + tv.tv_usec * 1e-3;
}

template <typename T>
static vector<T> load(const char* path, size_t n)
{
    vector<T> v(n);
    FILE* f = fopen(path, "rb");
    if (!f) { fprintf(stderr, "cannot open %s\n", path); exit(2); }
    if (fread(v.data(), sizeof(T), n, f) != n) { fprintf(stderr, "short read %s\n", path); exit(2); }
    fclose(f);
    return v;
}

template <typename T>
static void save(const char* path, const vector<T>& v)
{
    FILE* f = fopen(path, "wb");
    if (!f) { fprintf(stderr, "cannot write %s\n", path); exit(2); }
    fwrite(v.data(), sizeof(T), v.size(), f);
    fclose(f);
}

static void vm_init()
{
    // Interpreter only: the OpenCL entry points all fail in the oracle build.
    istringstream spec("EnableInterpreter\n");
    init(spec);
}

// C = matmul(A, B); s = sum(C * C)          (512x512 matmul trace)
static int cmd_matmul_sum(int argc, char** argv)
{
    if (argc < 7) return 1;
    const size_t n = atol(argv[2]);
    vector<float> A = load<float>(argv[3], n * n), B = load<float>(argv[4], n * n);
    vector<float> C(n * n);
    const double t0 = now_ms();
    Arrayf32 a = make2(n, n, A.data());
    Arrayf32 b = make2(n, n, B.data());
    Arrayf32 c = matmul(a, b);
    Arrayf32 s = sum(c * c);
    const float sv = s.read_scalar();
    c.read1(C.data(), n * n * sizeof(float));
    const double t1 = now_ms();
    save(argv[5], C);
    printf("ms=%.3f s=%.9g\n", t1 - t0, sv);
    FILE* f = fopen(argv[6], "w"); fprintf(f, "%.9g\n", sv); fclose(f);
    return 0;
}

// C = matmul(A, B) with A MxK, B KxN (row-major, W = columns, H = rows)
template <typename T, typename ARR>
static int gemm_t(int argc, char** argv)
{
    if (argc < 8) return 1;
    const size_t M = atol(argv[2]), N = atol(argv[3]), K = atol(argv[4]);
    vector<T> A = load<T>(argv[5], M * K), B = load<T>(argv[6], K * N);
    vector<T> C(M * N);
    const double t0 = now_ms();
    ARR a = make2(K, M, A.data());
    ARR b = make2(N, K, B.data());
    ARR c = matmul(a, b);
    c.read1(C.data(), M * N * sizeof(T));
    const double t1 = now_ms();
    save(argv[7], C);
    printf("ms=%.3f\n", t1 - t0);
    return 0;
}

// y = matmul(A, x) with A MxN matrix, x length-N vector
template <typename T, typename ARR>
static int gemv_t(int argc, char** argv)
{
    if (argc < 7) return 1;
    const size_t M = atol(argv[2]), N = atol(argv[3]);
    vector<T> A = load<T>(argv[4], M * N), x = load<T>(argv[5], N);
    vector<T> y(M);
    const double t0 = now_ms();
    ARR a = make2(N, M, A.data());
    ARR v = make1(N, x.data());
    ARR r = matmul(a, v);
    r.read1(y.data(), M * sizeof(T));
    const double t1 = now_ms();
    save(argv[6], y);
    printf("ms=%.3f\n", t1 - t0);
    return 0;
}

// payoff = mean(max(S - 100, 0)), S = 100 * exp(drift + 0.2 * Z), Z given
static int cmd_mc(int argc, char** argv)
{
    if (argc < 4) return 1;
    const size_t n = atol(argv[2]);
    vector<float> Z = load<float>(argv[3], n);
    const double t0 = now_ms();
    Arrayf32 z = make1(n, Z.data());
    Arrayf32 S = 100.0f * exp((0.05f - 0.5f * 0.2f * 0.2f) * 1.0f + 0.2f * z);
    Arrayf32 payoff = mean(chai::max(S - 100.0f, 0.0f));
    const float p = payoff.read_scalar();
    const double t1 = now_ms();
    printf("ms=%.3f payoff=%.9g\n", t1 - t0, p);
    return 0;
}

// Same trace with the interpreter's own normal generator (timing baseline).
static int cmd_mc_rng(int argc, char** argv)
{
    if (argc < 4) return 1;
    const size_t W = atol(argv[2]), H = atol(argv[3]);
    RNGf32 g(RNG_PHILOX, 42);
    const double t0 = now_ms();
    Arrayf32 z = rng_normal_make(g, W, H);
    Arrayf32 S = 100.0f * exp((0.05f - 0.5f * 0.2f * 0.2f) * 1.0f + 0.2f * z);
    Arrayf32 payoff = mean(chai::max(S - 100.0f, 0.0f));
    const float p = payoff.read_scalar();
    const double t1 = now_ms();
    printf("ms=%.3f payoff=%.9g\n", t1 - t0, p);
    return 0;
}

// 8-direction Kirsch compass filter through gather2_floor with periodic wrap.
static int cmd_kirsch(int argc, char** argv)
{
    if (argc < 6) return 1;
    const size_t W = atol(argv[2]), H = atol(argv[3]);
    vector<float> img = load<float>(argv[4], W * H);
    vector<float> out(W * H);
    const double t0 = now_ms();
    Arrayf32 A = make2(W, H, img.data());
    Arrayf32 X = index_f32(0, W, H);
    Arrayf32 Y = index_f32(1, W, H);
    // neighbours clockwise from north-west
    Arrayf32 n0 = gather2_floor(A, X - 1, Y - 1);
    Arrayf32 n1 = gather2_floor(A, X, Y - 1);
    Arrayf32 n2 = gather2_floor(A, X + 1, Y - 1);
    Arrayf32 n3 = gather2_floor(A, X + 1, Y);
    Arrayf32 n4 = gather2_floor(A, X + 1, Y + 1);
    Arrayf32 n5 = gather2_floor(A, X, Y + 1);
    Arrayf32 n6 = gather2_floor(A, X - 1, Y + 1);
    Arrayf32 n7 = gather2_floor(A, X - 1, Y);
    Arrayf32 total = n0 + n1 + n2 + n3 + n4 + n5 + n6 + n7;
    // response k = 5 * (three consecutive neighbours) - 3 * (other five)
    //            = 8 * (three consecutive) - 3 * total
    Arrayf32 r0 = 8.0f * (n0 + n1 + n2) - 3.0f * total;
    Arrayf32 r1 = 8.0f * (n1 + n2 + n3) - 3.0f * total;
    Arrayf32 r2 = 8.0f * (n2 + n3 + n4) - 3.0f * total;
    Arrayf32 r3 = 8.0f * (n3 + n4 + n5) - 3.0f * total;
    Arrayf32 r4 = 8.0f * (n4 + n5 + n6) - 3.0f * total;
    Arrayf32 r5 = 8.0f * (n5 + n6 + n7) - 3.0f * total;
    Arrayf32 r6 = 8.0f * (n6 + n7 + n0) - 3.0f * total;
    Arrayf32 r7 = 8.0f * (n7 + n0 + n1) - 3.0f * total;
    Arrayf32 K = chai::max(chai::max(chai::max(r0, r1), chai::max(r2, r3)),
                           chai::max(chai::max(r4, r5), chai::max(r6, r7)));
    K.read1(out.data(), W * H * sizeof(float));
    const double t1 = now_ms();
    save(argv[5], out);
    printf("ms=%.3f\n", t1 - t0);
    return 0;
}

// sum / mean / dot_product of given f32 arrays (reduction semantics)
static int cmd_reduce(int argc, char** argv)
{
    if (argc < 5) return 1;
    const size_t W = atol(argv[2]), H = atol(argv[3]);
    vector<float> a = load<float>(argv[4], W * H);
    vector<float> b = argc > 5 ? load<float>(argv[5], W * H) : a;
    const double t0 = now_ms();
    Arrayf32 A = make2(W, H, a.data());
    Arrayf32 B = make2(W, H, b.data());
    Arrayf32 S = sum(A), Mn = mean(A), D = dot_product(A, B);
    const float s = S.read_scalar();
    const float m = Mn.read_scalar();
    const float d = D.read_scalar();
    const double t1 = now_ms();
    printf("ms=%.3f sum=%.9g mean=%.9g dot=%.9g\n", t1 - t0, s, m, d);
    return 0;
}

int main(int argc, char** argv)
{
    if (argc < 2) { fprintf(stderr, "usage: ref_driver <cmd> ...\n"); return 1; }
    vm_init();
    const string cmd = argv[1];
    int rc = 1;
    if (cmd == "matmul_sum") rc = cmd_matmul_sum(argc, argv);
    else if (cmd == "gemm_f32") rc = gemm_t<float, Arrayf32>(argc, argv);
    else if (cmd == "gemm_f64") rc = gemm_t<double, Arrayf64>(argc, argv);
    else if (cmd == "gemv_f32") rc = gemv_t<float, Arrayf32>(argc, argv);
    else if (cmd == "gemv_f64") rc = gemv_t<double, Arrayf64>(argc, argv);
    else if (cmd == "mc") rc = cmd_mc(argc, argv);
    else if (cmd == "mc_rng") rc = cmd_mc_rng(argc, argv);
    else if (cmd == "kirsch") rc = cmd_kirsch(argc, argv);
    else if (cmd == "reduce") rc = cmd_reduce(argc, argv);
    else fprintf(stderr, "unknown command %s\n", argv[1]);
    shutdown();
    return rc;
}
