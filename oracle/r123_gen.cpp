// Prints the Random123 OpenCL source that the reference JIT generates
// (Random123/Random123.cpp:100-130 driving R123Philox::print and
// R123Threefry::print) for both generator families, 32- and 64-bit words and
// vector lengths 2 and 4.  build_ref.py keeps the bijections of that text and
// compiles them as C++, so the oracle's restatement is compared with the
// reference's own generated generators.
//
// Test infrastructure only; the product never links or runs this program.
#include <iostream>

#include "Random123.hpp"

int main()
{
    chai_internal::Random123 r;
    r.prec32();
    r.prec64();
    r.vecLength2();
    r.vecLength4();
    r.philox();
    r.threefry();
    r.print(std::cout);
    std::cout << std::endl;
    return 0;
}
