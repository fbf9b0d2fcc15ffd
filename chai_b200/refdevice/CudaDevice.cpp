// CudaDevice: a VectorTrace of the reference runtime evaluated by chai_b200.
//
// Per trace (sub_evaluate):
//   1. every statement's bytecode stack (Stak<BC>, pushed last argument first,
//      opcode last: api/ArrayFun.cpp:44-52) becomes the chai_bc cells of a
//      chai_stmt in the same order; an array memory box (a BC pointer cell
//      holding the absolute statement index, common/ClientTrace.cpp:286-293)
//      becomes a MEMORY cell naming a device buffer -- the box's host data
//      uploaded for make1/make2, an empty buffer the back end fills for
//      read_scalar/read1/read2 -- or, for ProgramCL, a KERNEL cell with the
//      AstOpenCL program, name, arguments and NDRange;
//   2. variables read from earlier traces are bound as inputs: a value this
//      device left resident is bound in place, anything else (a make box, a
//      value another device computed) is uploaded;
//   3. variables the trace leaves live (VectorTrace::liveVariables) are bound
//      as outputs to fresh device buffers; after the evaluation each gets a
//      host BackMem whose rows carry the reference's width padding, filled
//      only when the host asks for it (swizzle), and its FrontMem boxes
//      become the variable's value (VectorNut::setNutMem, as
//      runtime/Interpreter.cpp:335-363 does);
//   4. read boxes are filled from their device buffers.
// A failure returns false: DeviceBase::evaluate frees the trace's boxes and
// the scheduler reports DEVICE_FAILURE (runtime/Executor.cpp:56-59).
#include "CudaDevice.hpp"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include <set>
#include <utility>
#include <vector>

#include "AstOpenCL.hpp"
#include "BackMem.hpp"
#include "ByteCodes.hpp"
#include "FrontMem.hpp"
#include "MemalignSTL.hpp"
#include "PrecType.hpp"
#include "VectorNut.hpp"

using namespace std;

namespace chai_internal {

namespace {

// Every BackMem this device creates reports to this forwarder, which lives
// until the process exits: a BackMem released after the device is gone (an
// array that outlives shutdown) finds no device and does nothing.
class CudaMemHub : public MemCallback
{
    pthread_mutex_t _mtx;
    CudaDevice*     _dev;

public:
    CudaMemHub(void) : _dev(NULL) { pthread_mutex_init(&_mtx, NULL); }

    void attach(CudaDevice* d)
    {
        pthread_mutex_lock(&_mtx);
        _dev = d;
        pthread_mutex_unlock(&_mtx);
    }

    void swizzle(BackMem* m)
    {
        pthread_mutex_lock(&_mtx);
        if (_dev) _dev->swizzle(m);
        pthread_mutex_unlock(&_mtx);
    }

    void untrackMem(BackMem* m)
    {
        pthread_mutex_lock(&_mtx);
        if (_dev) _dev->untrackMem(m);
        pthread_mutex_unlock(&_mtx);
    }
};

CudaMemHub& hub(void)
{
    static CudaMemHub h;
    return h;
}

size_t elemBytes(const size_t prec) { return PrecType::sizeOf(prec); }

// Dense slots x H x W device layout <-> host boxes whose rows are
// PrecType::padWidth(prec, W) elements.  A box list shorter than `slots` is
// repeated (one make box shared by every trace of a vector trace).
void packBoxes(const vector< FrontMem* >& boxes, const size_t slots, const size_t prec, const size_t W,
               const size_t H, vector< char >& dense)
{
    const size_t eb = elemBytes(prec), pw = PrecType::padWidth(prec, W);
    dense.resize(slots * H * W * eb);
    for (size_t s = 0; s < slots; s++)
    {
        const char* src = static_cast< const char* >(boxes[s % boxes.size()]->ptrMem());
        char* dst = &dense[0] + s * H * W * eb;
        for (size_t y = 0; y < H; y++) memcpy(dst + y * W * eb, src + y * pw * eb, W * eb);
    }
}

void unpackBoxes(const vector< char >& dense, const size_t slots, const size_t prec, const size_t W,
                 const size_t H, const vector< FrontMem* >& boxes)
{
    const size_t eb = elemBytes(prec), pw = PrecType::padWidth(prec, W);
    for (size_t s = 0; s < slots && s < boxes.size(); s++)
    {
        char* dst = static_cast< char* >(boxes[s]->ptrMem());
        const char* src = &dense[0] + s * H * W * eb;
        for (size_t y = 0; y < H; y++) memcpy(dst + y * pw * eb, src + y * W * eb, W * eb);
    }
}

struct ReadBox
{
    uint64_t             id;
    vector< FrontMem* >  boxes;
    size_t               prec, W, H;
};

// Flattens one statement's bytecode into chai_bc cells and collects what the
// trace needs bound or uploaded.
class Flattener : public Visit< BC >
{
public:
    VectorTrace&                           vt;
    CudaDevice&                            dev;
    chai_cuda_ctx*                         ctx;
    const size_t                           slots;
    vector< chai_bc >*                     cells;
    set< pair< uint32_t, uint32_t > >&     assigned;     // (variable, version) set by earlier statements
    map< uint32_t, uint32_t >&             latest;       // variable -> version last set in this trace
    const set< uint32_t >&                 written;      // variables this trace assigns
    map< uint32_t, chai_buffer_binding >&  inputs;
    vector< uint64_t >&                    scratch;      // buffers released after the trace
    vector< ReadBox >&                     reads;
    vector< chai_inline_kernel >&          kernels;
    vector< vector< chai_kernel_arg > >&   kernelArgs;
    vector< string >&                      kernelText;
    string                                 error;
    size_t                                 current;      // statement being flattened
    bool                                   makeSlots;    // the next scalar is a make statement's slot count

    Flattener(VectorTrace& v, CudaDevice& d, chai_cuda_ctx* c, size_t s, set< pair< uint32_t, uint32_t > >& a,
              map< uint32_t, uint32_t >& l, const set< uint32_t >& w, map< uint32_t, chai_buffer_binding >& in,
              vector< uint64_t >& sc, vector< ReadBox >& rd, vector< chai_inline_kernel >& k,
              vector< vector< chai_kernel_arg > >& ka, vector< string >& kt)
        : vt(v), dev(d), ctx(c), slots(s), cells(NULL), assigned(a), latest(l), written(w), inputs(in),
          scratch(sc), reads(rd), kernels(k), kernelArgs(ka), kernelText(kt), current(0), makeSlots(false) { }

    void push(const uint32_t kind, const uint32_t code, const uint32_t version, const double scalar,
              const uint64_t buffer)
    {
        chai_bc b;
        memset(&b, 0, sizeof b);
        b.kind = kind;
        b.code = code;
        b.version = version;
        b.scalar = scalar;
        b.buffer = buffer;
        cells->push_back(b);
    }

    // A variable's value from an earlier trace, bound as an input.
    void bindInput(const uint32_t variable, const uint32_t version)
    {
        if (inputs.count(variable) || !error.empty()) return;
        if (0 == vt.vectorNuts().count(variable))
        {
            error = "variable without a value";
            return;
        }
        const vector< FrontMem* > fm = vt.vectorNuts()[variable]->getNutMem(version);
        if (fm.empty() || NULL == fm.front()->ptrMem())
        {
            error = "variable without array memory";
            return;
        }
        const FrontMem* f0 = fm.front();
        const size_t prec = f0->prec(), W = f0->W(), H = f0->H();
        chai_buffer_binding b;
        memset(&b, 0, sizeof b);
        b.variable = variable;
        b.prec = (uint32_t)prec;
        b.width = W;
        b.height = H;
        b.slots = (uint32_t)slots;
        // resident here, one buffer with every slot in order: bind it (a copy
        // when this trace assigns the variable, so the earlier value survives)
        CudaDevice::Resident r;
        BackMem* bm = f0->getBackMem();
        bool whole = bm && dev.lookupResident(bm, r) && r.slots == slots && r.prec == prec && r.W == W && r.H == H &&
                     fm.size() == slots;
        const size_t slotBytes = PrecType::padWidth(prec, W) * H * elemBytes(prec);
        for (size_t s = 0; whole && s < fm.size(); s++)
            whole = fm[s]->getBackMem() == bm &&
                    static_cast< char* >(fm[s]->ptrMem()) == static_cast< char* >(bm->ptrMem()) + s * slotBytes;
        const size_t bytes = slots * H * W * elemBytes(prec);
        if (whole)
        {
            if (written.count(variable))
            {
                b.buffer = dev.newId();
                if (ctx && chai_cuda_buffer_copy(ctx, b.buffer, r.id, bytes)) error = chai_cuda_last_error(ctx);
                scratch.push_back(b.buffer);
            }
            else
            {
                b.buffer = r.id;
            }
        }
        else
        {
            // host values: a value resident here is read back first
            for (size_t s = 0; s < fm.size(); s++)
                if (fm[s]->getBackMem()) fm[s]->getBackMem()->swizzle();
            vector< char > dense;
            packBoxes(fm, slots, prec, W, H, dense);
            b.buffer = dev.newId();
            if (ctx && chai_cuda_upload(ctx, b.buffer, dense.empty() ? NULL : &dense[0], dense.size()))
                error = chai_cuda_last_error(ctx);
            scratch.push_back(b.buffer);
        }
        inputs[variable] = b;
    }

    void visit(const uint32_t variable, const uint32_t version)
    {
        push(CHAI_BC_VARIABLE, variable, version, 0, 0);
        if (!assigned.count(make_pair(variable, version)) && !latest.count(variable))
            bindInput(variable, version);
    }

    void visit(const uint32_t opCode) { push(CHAI_BC_OPCODE, opCode, 0, 0, 0); }

    void visit(const double scalar)
    {
        // a make statement of a vector trace that gathers single traces
        // (Scheduler batching, runtime/Scheduler.cpp:48-89) holds one box per
        // trace: its slot count is the number of traces
        const double v = makeSlots ? (scalar > (double)slots ? scalar : (double)slots) : scalar;
        makeSlots = false;
        push(CHAI_BC_SCALAR, 0, 0, v, 0);
    }

    void visit(void* ptr)
    {
        const size_t stmtIndex = reinterpret_cast< size_t >(ptr);
        if (0 == vt.frontMem().count(stmtIndex) || vt.frontMem()[stmtIndex].empty())
        {
            error = "array memory box missing";
            return;
        }
        const vector< FrontMem* >& boxes = vt.frontMem()[stmtIndex];
        const FrontMem* proto = boxes.front();
        if (0 == proto->W() && 0 == proto->H())
        {
            inlineKernel(static_cast< AstOpenCL* >(proto->dataPtr()));
            return;
        }
        const uint64_t id = dev.newId();
        scratch.push_back(id);
        if (proto->dataPtr())
        {
            // make1 / make2: the box data (memalloc copied it into padded rows);
            // the next cell is the statement's slot count
            makeSlots = slots > 1;
            vector< char > dense;
            packBoxes(boxes, slots, proto->prec(), proto->W(), proto->H(), dense);
            if (ctx && chai_cuda_upload(ctx, id, dense.empty() ? NULL : &dense[0], dense.size()))
                error = chai_cuda_last_error(ctx);
        }
        else
        {
            // read_scalar / read1 / read2: filled by the back end
            ReadBox rb;
            rb.id = id;
            rb.boxes = boxes;
            rb.prec = proto->prec();
            rb.W = proto->W();
            rb.H = proto->H();
            reads.push_back(rb);
        }
        push(CHAI_BC_MEMORY, 0, 0, 0, id);
    }

    // ProgramCL (api/ProgramCL.cpp:213-226; arguments read by their declared
    // precision as enqueue/EnqueueAST.cpp:432-474 does)
    void inlineKernel(AstOpenCL* ast)
    {
        if (!ast)
        {
            error = "inline kernel without a program";
            return;
        }
        string text;
        for (size_t i = 0; i < ast->programSource().size(); i++) (text += ast->programSource()[i]) += "\n";
        kernelText.push_back(text);
        kernelText.push_back(ast->kernelName());
        vector< chai_kernel_arg > args;
        for (size_t i = 0; i < ast->getNumArgs(); i++)
        {
            chai_kernel_arg a;
            memset(&a, 0, sizeof a);
            a.prec = (uint32_t)ast->getArgPrec(i);
            if (ast->isArgArray(i))
            {
                a.kind = CHAI_KARG_ARRAY;
                a.variable = ast->getArgUInt32(i);
                // the array's current version: set earlier in this trace, else
                // the one later statements of the trace read
                if (latest.count(a.variable))
                {
                    a.version = latest[a.variable];
                }
                else if (!laterVersion(a.variable, a.version))
                {
                    error = "inline kernel array argument not read in its trace";
                    return;
                }
                else
                {
                    bindInput(a.variable, a.version);
                }
            }
            else if (ast->isArgLocal(i))
            {
                a.kind = CHAI_KARG_LOCAL;
                a.value = (double)ast->getArgSizeT(i);
            }
            else
            {
                a.kind = CHAI_KARG_SCALAR;
                switch (a.prec)
                {
                    case (PrecType::UInt32) : a.value = ast->getArgUInt32(i); break;
                    case (PrecType::Int32) : a.value = ast->getArgInt32(i); break;
                    case (PrecType::Float) : a.value = ast->getArgFloat(i); break;
                    default : a.value = ast->getArgDouble(i); break;
                }
            }
            args.push_back(a);
        }
        kernelArgs.push_back(args);
        chai_inline_kernel k;
        memset(&k, 0, sizeof k);
        k.n_args = (uint32_t)args.size();
        const bool twoD = ast->getWorkDim() > 1;
        k.global_size[0] = ast->getGlobalWorkDim(0);
        k.local_size[0] = ast->getLocalWorkDim(0);
        k.global_size[1] = twoD ? ast->getGlobalWorkDim(1) : 0;
        k.local_size[1] = twoD ? ast->getLocalWorkDim(1) : 0;
        kernels.push_back(k);       // text, name and argument pointers are set once the lists stop growing
        push(CHAI_BC_KERNEL, 0, 0, 0, kernels.size() - 1);
    }

    // version of `variable` the first later statement reads
    bool laterVersion(const uint32_t variable, uint32_t& version);
};

class VersionFinder : public Visit< BC >
{
public:
    uint32_t variable, version;
    bool     found;
    VersionFinder(uint32_t v) : variable(v), version(0), found(false) { }
    void visit(const uint32_t var, const uint32_t ver)
    {
        if (!found && var == variable)
        {
            found = true;
            version = ver;
        }
    }
    void visit(const uint32_t) { }
    void visit(const double) { }
    void visit(void*) { }
};

bool Flattener::laterVersion(const uint32_t variable, uint32_t& version)
{
    for (size_t i = current + 1; i < vt.traceLength(); i++)
    {
        VersionFinder f(variable);
        vt.getRHS(i).ascend(f);
        if (f.found)
        {
            version = f.version;
            return true;
        }
    }
    return false;
}

// CHAI_CUDA_TRACE=1: each trace as the back end receives it, on stderr (the
// counterpart of the reference's logged kernel source, kernel/KernelCache.cpp:82-89)
void dumpTrace(const chai_trace_desc& d, const vector< chai_buffer_binding >& binds,
               const vector< chai_value_shape >& shapes, size_t nshapes)
{
    fprintf(stderr, "trace %llx: %u statements, %u traces\n", (unsigned long long)d.hash, d.n_stmts, d.num_traces);
    for (uint32_t i = 0; i < d.n_stmts; i++)
    {
        const chai_stmt& st = d.stmts[i];
        fprintf(stderr, "  (%u,%u) =", st.lhs_variable, st.lhs_version);
        for (uint32_t c = 0; c < st.n_cells; c++)
        {
            const chai_bc& b = st.cells[c];
            switch (b.kind)
            {
                case CHAI_BC_OPCODE : fprintf(stderr, " op%u", b.code); break;
                case CHAI_BC_VARIABLE : fprintf(stderr, " v%u.%u", b.code, b.version); break;
                case CHAI_BC_SCALAR : fprintf(stderr, " %g", b.scalar); break;
                case CHAI_BC_MEMORY : fprintf(stderr, " mem#%llu", (unsigned long long)b.buffer); break;
                default : fprintf(stderr, " kernel#%llu", (unsigned long long)b.buffer); break;
            }
        }
        fprintf(stderr, "\n");
    }
    for (size_t i = 0; i < binds.size(); i++)
        fprintf(stderr, "  bind v%u prec %u %llux%llu x%u -> #%llu\n", binds[i].variable, binds[i].prec,
                (unsigned long long)binds[i].width, (unsigned long long)binds[i].height, binds[i].slots,
                (unsigned long long)binds[i].buffer);
    for (size_t i = 0; i < nshapes && i < shapes.size(); i++)
        fprintf(stderr, "  value v%u.%u prec %u %llux%llu x%u\n", shapes[i].variable, shapes[i].version,
                shapes[i].prec, (unsigned long long)shapes[i].width, (unsigned long long)shapes[i].height,
                shapes[i].slots);
}

} // namespace

CudaDevice::CudaDevice(const int deviceNum, const string& config)
    : DeviceBase(deviceNum),
      _ctx(NULL),
      _nextId(1ull << 40),
      _failures(0)
{
    pthread_mutex_init(&_mtx, NULL);
    const int st = chai_cuda_init(deviceNum < 0 ? 0 : deviceNum, config.c_str(), &_ctx);
    if (st)
    {
        fprintf(stderr, "CudaDevice: chai_cuda_init failed: %s\n", chai_cuda_error_string(st));
        _ctx = NULL;
    }
    hub().attach(this);
}

CudaDevice::~CudaDevice(void)
{
    hub().attach(NULL);
    if (_ctx) chai_cuda_shutdown(_ctx);      // frees every device buffer and module
    pthread_mutex_destroy(&_mtx);
}

bool CudaDevice::ok(void) const { return NULL != _ctx; }

uint64_t CudaDevice::newId(void)
{
    pthread_mutex_lock(&_mtx);
    const uint64_t id = _nextId++;
    pthread_mutex_unlock(&_mtx);
    return id;
}

bool CudaDevice::lookupResident(BackMem* m, Resident& r)
{
    pthread_mutex_lock(&_mtx);
    map< BackMem*, Resident >::const_iterator it = _resident.find(m);
    const bool hit = it != _resident.end();
    if (hit) r = it->second;
    pthread_mutex_unlock(&_mtx);
    return hit;
}

// Host BackMem for a live variable whose value stays in device buffer `id`:
// padded rows, zero-filled, read back on swizzle; one FrontMem per slot
// (memmgr/MemBase.cpp allocates the interpreter's values the same way).
BackMem* CudaDevice::residentValue(const chai_value_shape& v, const uint64_t id, vector< FrontMem* >& fronts)
{
    const size_t prec = v.prec, W = v.width, H = v.height, slots = v.slots;
    const size_t slotBytes = PrecType::padWidth(prec, W) * H * elemBytes(prec);
    void* host = NULL;
    if (0 != posix_memalign(&host, MEMORY_ALIGNMENT, slotBytes * slots)) return NULL;
    memset(host, 0, slotBytes * slots);
    BackMem* bm = NULL;
    switch (prec)
    {
        case (PrecType::UInt32) :
            bm = new BackMem(W, H, slots, slots, static_cast< uint32_t* >(host), &hub()); break;
        case (PrecType::Int32) :
            bm = new BackMem(W, H, slots, slots, static_cast< int32_t* >(host), &hub()); break;
        case (PrecType::Float) :
            bm = new BackMem(W, H, slots, slots, static_cast< float* >(host), &hub()); break;
        default :
            bm = new BackMem(W, H, slots, slots, static_cast< double* >(host), &hub()); break;
    }
    for (size_t s = 0; s < slots; s++)
    {
        FrontMem* f = NULL;
        switch (prec)
        {
            case (PrecType::UInt32) : f = new FrontMem(W, H, static_cast< uint32_t* >(NULL)); break;
            case (PrecType::Int32) : f = new FrontMem(W, H, static_cast< int32_t* >(NULL)); break;
            case (PrecType::Float) : f = new FrontMem(W, H, static_cast< float* >(NULL)); break;
            default : f = new FrontMem(W, H, static_cast< double* >(NULL)); break;
        }
        f->setBackMem(static_cast< char* >(host) + s * slotBytes, bm);
        fronts.push_back(f);
    }
    // the front boxes own the backing memory
    bm->release();
    Resident r;
    r.id = id;
    r.prec = prec;
    r.W = W;
    r.H = H;
    r.slots = slots;
    pthread_mutex_lock(&_mtx);
    _resident[bm] = r;
    pthread_mutex_unlock(&_mtx);
    return bm;
}

bool CudaDevice::sub_evaluate(VectorTrace& vt)
{
    const char* traceEnv = getenv("CHAI_CUDA_TRACE");
    const bool dump = traceEnv && *traceEnv && traceEnv[0] != '0';
    if (!_ctx && !dump) return fail("no CUDA context");
    const size_t n = vt.traceLength();
    const size_t slots = vt.numTraces() ? vt.numTraces() : 1;

    // constructor and destructor records of the client trace are statements
    // with no bytecode (ClientTrace constructor / destructor); the
    // interpreter skips them (runtime/Interpreter.cpp:340-356) and so does
    // this device
    set< uint32_t > written;
    for (size_t i = 0; i < n; i++)
        if (vt.getRHS(i).size()) written.insert(vt.getVariable(i));

    vector< vector< chai_bc > >          cells(n);
    vector< chai_stmt >                  stmts(n);
    set< pair< uint32_t, uint32_t > >    assigned;
    map< uint32_t, uint32_t >            latest;
    map< uint32_t, chai_buffer_binding > inputs;
    vector< uint64_t >                   scratch;
    vector< ReadBox >                    reads;
    vector< chai_inline_kernel >         kernels;
    vector< vector< chai_kernel_arg > >  kernelArgs;
    vector< string >                     kernelText;

    Flattener fl(vt, *this, _ctx, slots, assigned, latest, written, inputs, scratch, reads, kernels, kernelArgs,
                 kernelText);
    for (size_t i = 0; i < n && fl.error.empty(); i++)
    {
        if (!vt.getRHS(i).size()) continue;
        fl.current = i;
        fl.cells = &cells[i];
        vt.getRHS(i).ascend(fl);
        assigned.insert(make_pair(vt.getVariable(i), vt.getVersion(i)));
        latest[vt.getVariable(i)] = vt.getVersion(i);
    }
    bool good = fl.error.empty();
    size_t ns = 0;
    for (size_t i = 0; i < n; i++)
    {
        if (cells[i].empty()) continue;
        memset(&stmts[ns], 0, sizeof stmts[ns]);
        stmts[ns].lhs_variable = vt.getVariable(i);
        stmts[ns].lhs_version = vt.getVersion(i);
        stmts[ns].n_cells = (uint32_t)cells[i].size();
        stmts[ns].cells = &cells[i][0];
        ns++;
    }
    for (size_t k = 0; k < kernels.size(); k++)
    {
        kernels[k].source = kernelText[2 * k].c_str();
        kernels[k].name = kernelText[2 * k + 1].c_str();
        kernels[k].args = kernelArgs[k].empty() ? NULL : &kernelArgs[k][0];
    }
    chai_trace_desc desc;
    memset(&desc, 0, sizeof desc);
    desc.num_traces = (uint32_t)slots;
    desc.n_stmts = (uint32_t)ns;
    desc.stmts = stmts.empty() ? NULL : &stmts[0];
    desc.hash = vt.hashCode();
    desc.kernels = kernels.empty() ? NULL : &kernels[0];
    desc.n_kernels = (uint32_t)kernels.size();

    // what each statement produces, to size the live variables' host memory
    vector< chai_buffer_binding > binds;
    for (map< uint32_t, chai_buffer_binding >::const_iterator it = inputs.begin(); it != inputs.end(); it++)
        binds.push_back(it->second);
    vector< chai_value_shape > shapes(ns + 1);
    size_t nshapes = 0;
    if (good && chai_cuda_trace_shapes(&desc, binds.empty() ? NULL : &binds[0], binds.size(), &shapes[0],
                                       shapes.size(), &nshapes))
    {
        fl.error = "trace_shapes failed";
        good = false;
    }
    // live variables this trace assigns: bound as outputs (an input binding of
    // the same variable already holds a fresh buffer that becomes the output)
    map< uint32_t, chai_value_shape > live;
    for (size_t i = 0; good && i < nshapes && i < shapes.size(); i++)
        if (vt.liveVariables().count(shapes[i].variable)) live[shapes[i].variable] = shapes[i];
    map< uint32_t, uint64_t > outId;
    for (map< uint32_t, chai_value_shape >::const_iterator it = live.begin(); it != live.end(); it++)
    {
        const uint32_t var = it->first;
        map< uint32_t, chai_buffer_binding >::iterator in = inputs.find(var);
        if (in != inputs.end())
        {
            outId[var] = in->second.buffer;                  // fresh: written variables get copies
            for (size_t b = 0; b < binds.size(); b++)
                if (binds[b].variable == var) binds[b].slots = it->second.slots;
            continue;
        }
        chai_buffer_binding b;
        memset(&b, 0, sizeof b);
        b.variable = var;
        b.prec = it->second.prec;
        b.width = it->second.width;
        b.height = it->second.height;
        b.slots = it->second.slots;
        b.buffer = newId();
        outId[var] = b.buffer;
        binds.push_back(b);
    }

    if (dump) dumpTrace(desc, binds, shapes, nshapes);
    if (!_ctx)
    {
        fl.error = "no CUDA context";
        good = false;
    }
    if (good && chai_cuda_evaluate(_ctx, &desc, binds.empty() ? NULL : &binds[0], binds.size()))
    {
        fl.error = chai_cuda_last_error(_ctx);
        good = false;
    }

    // live values: resident buffers behind fresh host boxes
    for (map< uint32_t, chai_value_shape >::const_iterator it = live.begin(); good && it != live.end(); it++)
    {
        const uint32_t var = it->first;
        vector< FrontMem* > fronts;
        if (!residentValue(it->second, outId[var], fronts))
        {
            fl.error = "host memory for a live variable";
            good = false;
            break;
        }
        // the buffer now belongs to the value: keep it past the scratch release
        for (size_t k = 0; k < scratch.size(); k++)
            if (scratch[k] == outId[var]) scratch[k] = 0;
        vt.vectorNuts()[var]->setNutMem(it->second.version, fronts);
    }
    // read boxes
    for (size_t r = 0; good && r < reads.size(); r++)
    {
        const ReadBox& rb = reads[r];
        vector< char > dense(slots * rb.H * rb.W * elemBytes(rb.prec));
        if (chai_cuda_readback(_ctx, rb.id, dense.empty() ? NULL : &dense[0], dense.size()))
        {
            fl.error = chai_cuda_last_error(_ctx);
            good = false;
            break;
        }
        unpackBoxes(dense, slots, rb.prec, rb.W, rb.H, rb.boxes);
    }
    if (_ctx)
        for (size_t k = 0; k < scratch.size(); k++)
            if (scratch[k]) chai_cuda_release(_ctx, scratch[k]);
    if (!good)
    {
        if (_ctx)
            for (map< uint32_t, uint64_t >::const_iterator it = outId.begin(); it != outId.end(); it++)
                chai_cuda_release(_ctx, it->second);
        return fail(fl.error);
    }
    _failures = 0;
    return true;
}

// A failed trace goes back to the scheduler's queue marked as failing on this
// device (DEVICE_FAILURE, runtime/Scheduler.cpp:221-252, 300-378), which
// never offers it to this device again.  With the CUDA device alone in the
// table nothing else would take it and the client would wait for ever, so
// the program stops with the reason.
bool CudaDevice::fail(const string& why)
{
    fprintf(stderr, "CudaDevice: trace failed: %s\n", why.c_str());
    ++_failures;
    fflush(stderr);
    _exit(70);          // no static destructors: the scheduler's threads are still running
    return false;
}

void CudaDevice::swizzle(BackMem* m)
{
    Resident r;
    if (!_ctx || !lookupResident(m, r)) return;
    vector< char > dense(r.slots * r.H * r.W * elemBytes(r.prec));
    if (chai_cuda_readback(_ctx, r.id, dense.empty() ? NULL : &dense[0], dense.size())) return;
    const size_t eb = elemBytes(r.prec), pw = PrecType::padWidth(r.prec, r.W);
    for (size_t s = 0; s < r.slots; s++)
    {
        char* dst = static_cast< char* >(m->ptrMem()) + s * pw * r.H * eb;
        const char* src = &dense[0] + s * r.H * r.W * eb;
        for (size_t y = 0; y < r.H; y++) memcpy(dst + y * pw * eb, src + y * r.W * eb, r.W * eb);
    }
}

void CudaDevice::untrackMem(BackMem* m)
{
    pthread_mutex_lock(&_mtx);
    map< BackMem*, Resident >::iterator it = _resident.find(m);
    const bool hit = it != _resident.end();
    const uint64_t id = hit ? it->second.id : 0;
    if (hit) _resident.erase(it);
    pthread_mutex_unlock(&_mtx);
    if (hit && _ctx) chai_cuda_release(_ctx, id);
}

}; // namespace chai_internal
