// Packing of concurrent solves' tensor-core applies into one launch (no
// reference counterpart; the reference solves one request per GMRES call,
// FarField.hpp:706-708).
//
// Contexts attached to one Packer submit the dense stage of each operator
// apply (device pointers of their mesh and blocks) instead of launching it.
// A submission waits until every context that is inside a solve has
// submitted too, or until `max_wait_us` has passed; then one of the waiting
// threads launches a packed kernel over all pending problems of a class on
// the packer's stream (after each problem's AvOp, via events) and every
// submitter's stream waits for it.  The solves' other kernels stay on their
// own streams, so they still overlap on the GPU.  Whole target blocks per
// CTA (launch_boundary_tc_packed) make each problem's result independent of
// the packing.
#pragma once
#include <condition_variable>
#include <mutex>
#include <string>
#include <vector>

#include "ops.cuh"

namespace baemm
{

class Packer
{
public:
    Packer(int device, int max_wait_us);
    ~Packer();
    Packer(const Packer &) = delete;
    Packer &operator=(const Packer &) = delete;
    // A solve starts / ends on an attached context: the packer waits for the
    // submissions of the solves in progress.
    void join();
    void leave();
    // The dense stage of `item` (ready on `caller` once the work enqueued so
    // far has run); returns once it is enqueued in a packed launch and
    // `caller` waits for that launch.  Called from the context's thread.
    void apply(const TcPackItem &item, const OpFlags &f, const TcTuning &tune, cudaStream_t caller);
    int device() const { return device_; }
    long long launches() const;
    long long problems() const;

private:
    struct Pending
    {
        TcPackItem item;
        OpFlags flags;
        TcTuning tune;
        int cls = 0;
        cudaEvent_t ready = nullptr, done = nullptr;
        bool launched = false;
        std::string error;
    };
    void launch_all_locked();
    cudaEvent_t take_event_locked();

    int device_;
    int max_wait_us_;
    cudaStream_t stream_ = nullptr;
    DevBuf<int> err_;
    TcPackScratch scratch_;
    mutable std::mutex mu_;
    std::condition_variable cv_;
    std::vector<Pending *> pending_;
    std::vector<cudaEvent_t> events_;
    int active_ = 0;
    long long launches_ = 0, problems_ = 0;
};

// Membership of one solve (join on construction, leave on destruction).
class PackerSession
{
public:
    explicit PackerSession(Packer *p) : p_(p)
    {
        if (p_) p_->join();
    }
    ~PackerSession()
    {
        if (p_) p_->leave();
    }
    PackerSession(const PackerSession &) = delete;
    PackerSession &operator=(const PackerSession &) = delete;

private:
    Packer *p_;
};

} // namespace baemm
