// The reference runtime's device table (class DeviceMap, runtime/DeviceMap.hpp)
// with the chai_b200 device added.  This file takes the place of the
// reference's runtime/DeviceMap.cpp when the reference is linked with
// chai_b200; every other reference file is used as it is.
//
// With CHAI_CUDA set in the environment (its value is the back end's
// configuration string, e.g. "GemmPrecision=auto", or "1"), device number 0 is
// a CudaDevice and the table holds nothing else, so the scheduler sends every
// trace to the B200.  Without it the table is what the reference builds: the
// interpreter as device -1 when the spec enables it
// (runtime/DeviceMap.cpp:12-23) and a Translator per OpenCL device
// (runtime/DeviceMap.cpp:25-36).
#include <stdlib.h>

#include <string>

#include "CudaDevice.hpp"
#include "DeviceMap.hpp"
#include "Interpreter.hpp"
#include "OCLhacks.hpp"
#include "Translator.hpp"

using namespace std;

namespace chai_internal {

DeviceMap::DeviceMap(OCLinit& oclInit, istream& configSpec)
{
    // the spec's hacks and device list are read first in every configuration
    OCLhacks::singleton().initHacks(oclInit, configSpec);

    const char* cuda = getenv("CHAI_CUDA");
    if (cuda && *cuda)
    {
        const string config = (string(cuda) == "1") ? string() : string(cuda);
        CudaDevice* dev = new CudaDevice(0, config);
        dev->initDevice();          // host boxes of make / read statements: MemInterp
        _deviceMap[0] = dev;
        _allDevnums.insert(0);
        return;
    }

    if (OCLhacks::singleton().enableInterpreter())
    {
        Interpreter* interp = new Interpreter(-1);
        interp->initDevice();
        _deviceMap[-1] = interp;
        _allDevnums.insert(-1);
    }

    const set< size_t >& ocl = OCLhacks::singleton().deviceIndexes();
    for (set< size_t >::const_iterator it = ocl.begin(); it != ocl.end(); ++it)
    {
        const int devnum = static_cast< int >(*it);
        Translator* jit = new Translator(devnum);
        jit->initDevice(oclInit);
        _deviceMap[devnum] = jit;
        _allDevnums.insert(devnum);
    }
}

DeviceMap::~DeviceMap(void)
{
    for (map< int, DeviceBase* >::iterator it = _deviceMap.begin(); it != _deviceMap.end(); ++it)
        delete it->second;
}

void DeviceMap::extendLanguage(const uint32_t opCode,
                               const BaseInterp& interpHandler,
                               const BaseTrans& jitHandler)
{
    // an interpreter takes the interpreter handler, a JIT device the JIT one;
    // the CUDA device accepts neither (DeviceBase's defaults decline)
    for (map< int, DeviceBase* >::iterator it = _deviceMap.begin(); it != _deviceMap.end(); ++it)
    {
        if (it->first < 0)
            it->second->extendLanguage(opCode, interpHandler);
        else
            it->second->extendLanguage(opCode, jitHandler);
    }
}

const set< int >& DeviceMap::allDevnums(void) const
{
    return _allDevnums;
}

DeviceBase* DeviceMap::getDevice(const int deviceNum)
{
    map< int, DeviceBase* >::iterator it = _deviceMap.find(deviceNum);
    return it == _deviceMap.end() ? NULL : it->second;
}

}; // namespace chai_internal
