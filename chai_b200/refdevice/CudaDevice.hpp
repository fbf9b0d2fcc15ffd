// CudaDevice: the reference runtime's device plug-in for the chai_b200 back end.
//
// The reference front end (api/, bytecode/, common/, runtime/Scheduler) records
// traces and hands each VectorTrace to a DeviceBase (runtime/DeviceBase.hpp:
// 22-61); DeviceBase::evaluate allocates the host boxes of make and read
// statements (memmgr/MemInterpAlloc.cpp:13-210) and calls sub_evaluate
// (runtime/DeviceBase.cpp:87-101).  CudaDevice::sub_evaluate flattens the
// trace into a chai_trace_desc and runs it through the C ABI of
// include/chai_b200.h: make boxes are uploaded, live variables stay resident in
// device buffers behind host BackMem objects that read back only when the host
// asks (MemCallback::swizzle, common/MemCallback.hpp:13-21), and read boxes are
// filled after the evaluation.  This file is compiled with the reference's own
// headers; nothing in the reference is edited.
#ifndef _CHAI_CUDA_DEVICE_HPP_
#define _CHAI_CUDA_DEVICE_HPP_

#include <pthread.h>
#include <stdint.h>

#include <map>
#include <string>
#include <vector>

#include "DeviceBase.hpp"
#include "MemCallback.hpp"
#include "chai_b200.h"

namespace chai_internal {

class CudaDevice : public DeviceBase
{
public:
    // a device buffer holding the value of one host BackMem: slots x H x W
    // elements, dense (the host rows carry the reference's width padding)
    struct Resident
    {
        uint64_t id;
        size_t   prec, W, H, slots;
    };

    CudaDevice(const int deviceNum, const std::string& config);
    ~CudaDevice(void);

    bool ok(void) const;
    bool sub_evaluate(VectorTrace&);

    // MemCallback role (through the process-wide forwarder every BackMem
    // created here points at): device -> host on demand, and release
    void swizzle(BackMem*);
    void untrackMem(BackMem*);

    // buffer ids handed to the back end, and the buffer behind a host BackMem
    uint64_t newId(void);
    bool lookupResident(BackMem*, Resident&);

private:
    chai_cuda_ctx*                 _ctx;
    uint64_t                       _nextId;
    pthread_mutex_t                _mtx;        // _nextId, _resident (client threads swizzle / release)
    std::map< BackMem*, Resident > _resident;
    int                            _failures;   // failed traces in a row

    bool fail(const std::string& why);
    BackMem* residentValue(const chai_value_shape&, const uint64_t id, std::vector< FrontMem* >& fronts);
};

}; // namespace chai_internal

#endif
