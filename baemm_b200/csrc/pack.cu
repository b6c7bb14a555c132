// Packer: one tensor-core launch for the concurrent solves' applies (pack.cuh).
#include "pack.cuh"

#include <chrono>
#include <map>

namespace baemm
{

Packer::Packer(int device, int max_wait_us) : device_(device), max_wait_us_(std::max(0, max_wait_us))
{
    DeviceScope scope(device);
    BAEMM_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    BAEMM_CUDA(cudaMemsetAsync(err_.reserve(1), 0, sizeof(int), stream_));
    BAEMM_CUDA(cudaStreamSynchronize(stream_));
}

Packer::~Packer()
{
    DeviceScope scope(device_);
    if (stream_) cudaStreamSynchronize(stream_);
    for (cudaEvent_t e : events_) cudaEventDestroy(e);
    if (stream_) cudaStreamDestroy(stream_);
}

void Packer::join()
{
    std::lock_guard<std::mutex> lock(mu_);
    ++active_;
}

void Packer::leave()
{
    std::lock_guard<std::mutex> lock(mu_);
    --active_;
    // the waiting submitters may now be all there is
    if (!pending_.empty() && (int)pending_.size() >= active_)
    {
        try
        {
            launch_all_locked();
        }
        catch (...)
        {
            // the submitters saw the error in their Pending; nothing to report here
        }
    }
}

long long Packer::launches() const
{
    std::lock_guard<std::mutex> lock(mu_);
    return launches_;
}

long long Packer::problems() const
{
    std::lock_guard<std::mutex> lock(mu_);
    return problems_;
}

cudaEvent_t Packer::take_event_locked()
{
    if (!events_.empty())
    {
        cudaEvent_t e = events_.back();
        events_.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    BAEMM_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    return e;
}

void Packer::apply(const TcPackItem &item, const OpFlags &f, const TcTuning &tune, cudaStream_t caller)
{
    Pending p;
    p.item = item;
    p.item.ch = tc_chunks_per_unit(item.wc, tune.chunks);
    p.flags = f;
    p.tune = tune;
    p.cls = tc_pack_class(f, item.wc, tune);
    {
        std::lock_guard<std::mutex> lock(mu_);
        p.ready = take_event_locked();
        p.done = take_event_locked();
    }
    BAEMM_CUDA(cudaEventRecord(p.ready, caller));
    std::unique_lock<std::mutex> lock(mu_);
    pending_.push_back(&p);
    if ((int)pending_.size() >= active_) launch_all_locked();
    else
    {
        const auto deadline = std::chrono::steady_clock::now() + std::chrono::microseconds(max_wait_us_);
        cv_.wait_until(lock, deadline, [&] { return p.launched; });
        if (!p.launched) launch_all_locked();
    }
    const std::string error = p.error;
    if (error.empty()) BAEMM_CUDA(cudaStreamWaitEvent(caller, p.done, 0));
    events_.push_back(p.ready);
    events_.push_back(p.done);
    if (!error.empty()) throw Error(BAEMM_ERR_CUDA, "packed launch failed: " + error);
}

void Packer::launch_all_locked()
{
    std::vector<Pending *> todo;
    todo.swap(pending_);
    std::map<int, std::vector<Pending *>> groups;
    for (Pending *q : todo) groups[q->cls].push_back(q);
    for (auto &g : groups)
    {
        try
        {
            std::vector<TcPackItem> items;
            for (Pending *q : g.second)
            {
                BAEMM_CUDA(cudaStreamWaitEvent(stream_, q->ready, 0));
                items.push_back(q->item);
            }
            const Pending &first = *g.second.front();
            launch_boundary_tc_packed(items.data(), (int)items.size(), first.flags, first.tune, scratch_, err_.p,
                                      stream_);
            for (Pending *q : g.second) BAEMM_CUDA(cudaEventRecord(q->done, stream_));
            ++launches_;
            problems_ += (long long)items.size();
        }
        catch (const std::exception &e)
        {
            for (Pending *q : g.second) q->error = e.what();
        }
        for (Pending *q : g.second) q->launched = true;
    }
    cv_.notify_all();
}

} // namespace baemm
