// VapourSynth API 4 plugin for the B200 BM3Dv2 library: registers
// core.vsfeel.BM3Dv2 with the reference's namespace, identifier and argument
// string (src/vsfeel.cpp:350-364, src/bm3d.cpp:1558-1574) and forwards every
// callback to the C ABI in vsfeel_bm3d.h:
//
//   BM3DCreate   (src/bm3d.cpp:1043-1552) -> vsfeel_bm3d_create
//   BM3DGetFrame (src/bm3d.cpp:698-1028)  -> vsfeel_bm3d_frame_range (arInitial),
//                                            vsfeel_bm3d_get_frame(_ref) (arAllFramesReady)
//   BM3DFree     (src/bm3d.cpp:1030-1037) -> vsfeel_bm3d_free
//
// Compiled only where the VapourSynth SDK header is installed
// (csrc/build.py: build_vs_shim); it links libvsfeel_bm3d.so, which it finds
// through its run path in the installed layout
// (site-packages/vapoursynth/plugins/vsfeel/ -> site-packages/vsfeel/).
//
// Validation and its messages live in the library (they follow BM3DCreate's
// order and wording), so the shim only moves the argument map into
// vsfeel_bm3d_args and reports the library's error string.
#include <VapourSynth4.h>

#include "vsfeel_bm3d.h"

#include <climits>
#include <cstdint>
#include <map>

namespace {

struct Filter {
    VSNode* node = nullptr;
    VSNode* ref = nullptr;  // the basic estimate for the final (Wiener) pass
    const VSVideoInfo* vi = nullptr;
    vsfeel_bm3d* ctx = nullptr;
};

int to_int(int64_t v) {
    return v > INT_MAX ? INT_MAX : (v < INT_MIN ? INT_MIN : static_cast<int>(v));
}

// element i of an optional array argument, read as the reference does: an
// absent element leaves the count where it is (the library fills it from
// the previous element)
void read_float_array(const VSAPI* vsapi, const VSMap* in, const char* key, float out[3],
                      int* count) {
    *count = 0;
    for (int i = 0; i < 3; ++i) {
        int err = 0;
        const double v = vsapi->mapGetFloat(in, key, i, &err);
        if (err) break;
        out[i] = static_cast<float>(v);
        *count = i + 1;
    }
}

void read_int_array(const VSAPI* vsapi, const VSMap* in, const char* key, int out[3], int* count) {
    *count = 0;
    for (int i = 0; i < 3; ++i) {
        int err = 0;
        const int64_t v = vsapi->mapGetInt(in, key, i, &err);
        if (err) break;
        out[i] = to_int(v);
        *count = i + 1;
    }
}

void read_int(const VSAPI* vsapi, const VSMap* in, const char* key, int* out, int* set) {
    int err = 0;
    const int64_t v = vsapi->mapGetInt(in, key, 0, &err);
    *set = err ? 0 : 1;
    *out = err ? 0 : to_int(v);
}

vsfeel_bm3d_video_info info_of(const VSVideoInfo* vi) {
    vsfeel_bm3d_video_info v{};
    v.width = vi->width;
    v.height = vi->height;
    v.num_frames = vi->numFrames;
    v.color_family = vi->format.colorFamily == cfGray
                         ? VSFEEL_CF_GRAY
                         : (vi->format.colorFamily == cfYUV ? VSFEEL_CF_YUV : 0);
    v.sample_type = vi->format.sampleType == stFloat ? VSFEEL_ST_FLOAT : VSFEEL_ST_INTEGER;
    v.bits_per_sample = vi->format.bitsPerSample;
    v.sub_sampling_w = vi->format.subSamplingW;
    v.sub_sampling_h = vi->format.subSamplingH;
    return v;
}

// The frames a get_frame call fetches, held until the library releases them.
struct Fetcher {
    const VSAPI* vsapi;
    VSFrameContext* fc;
    VSNode* nodes[2];
    std::multimap<int, const VSFrame*> held[2];

    const float* fetch(int clip, int n, ptrdiff_t* stride) {
        const VSFrame* f = vsapi->getFrameFilter(n, nodes[clip], fc);
        if (!f) return nullptr;
        held[clip].emplace(n, f);
        *stride = vsapi->getStride(f, 0);
        return reinterpret_cast<const float*>(vsapi->getReadPtr(f, 0));
    }
    void release(int clip, int n) {
        auto it = held[clip].find(n);
        if (it == held[clip].end()) return;
        vsapi->freeFrame(it->second);
        held[clip].erase(it);
    }
    ~Fetcher() {
        for (auto& h : held)
            for (auto& kv : h) vsapi->freeFrame(kv.second);
    }
};

const float* fetch1(void* user, int n, ptrdiff_t* stride) {
    return static_cast<Fetcher*>(user)->fetch(0, n, stride);
}
void release1(void* user, int n) { static_cast<Fetcher*>(user)->release(0, n); }
const float* fetch2(void* user, int clip, int n, ptrdiff_t* stride) {
    return static_cast<Fetcher*>(user)->fetch(clip, n, stride);
}
void release2(void* user, int clip, int n) { static_cast<Fetcher*>(user)->release(clip, n); }

const VSFrame* VS_CC bm3d_get_frame(int n, int activation, void* instance, void** frame_data,
                                    VSFrameContext* fc, VSCore* core, const VSAPI* vsapi) {
    (void)frame_data;
    auto* d = static_cast<Filter*>(instance);
    if (activation == arInitial) {
        int first = n, last = n;
        if (vsfeel_bm3d_frame_range(d->ctx, n, &first, &last) != VSFEEL_OK) {
            vsapi->setFilterError(vsfeel_bm3d_last_error(), fc);
            return nullptr;
        }
        for (int f = first; f <= last; ++f) {
            vsapi->requestFrameFilter(f, d->node, fc);
            if (d->ref) vsapi->requestFrameFilter(f, d->ref, fc);
        }
        return nullptr;
    }
    if (activation != arAllFramesReady) return nullptr;

    // chroma planes of a YUV clip are referenced from the source frame
    // (zero-copy, src/bm3d.cpp:715-729); luma is written by the library
    const VSFrame* src = vsapi->getFrameFilter(n, d->node, fc);
    const VSFrame* plane_src[3] = {nullptr, src, src};
    const int planes[3] = {0, 1, 2};
    VSFrame* dst = vsapi->newVideoFrame2(&d->vi->format, d->vi->width, d->vi->height,
                                         d->vi->format.numPlanes > 1 ? plane_src : nullptr,
                                         d->vi->format.numPlanes > 1 ? planes : nullptr, src, core);
    int rc;
    {
        Fetcher fetcher{vsapi, fc, {d->node, d->ref}, {}};
        float* out = reinterpret_cast<float*>(vsapi->getWritePtr(dst, 0));
        const ptrdiff_t stride = vsapi->getStride(dst, 0);
        rc = d->ref ? vsfeel_bm3d_get_frame_ref(d->ctx, n, fetch2, release2, &fetcher, out, stride)
                    : vsfeel_bm3d_get_frame(d->ctx, n, fetch1, release1, &fetcher, out, stride);
    }
    vsapi->freeFrame(src);
    if (rc != VSFEEL_OK) {
        vsapi->setFilterError(vsfeel_bm3d_last_error(), fc);
        vsapi->freeFrame(dst);
        return nullptr;
    }
    return dst;
}

void VS_CC bm3d_free(void* instance, VSCore* core, const VSAPI* vsapi) {
    (void)core;
    auto* d = static_cast<Filter*>(instance);
    vsfeel_bm3d_free(d->ctx);
    vsapi->freeNode(d->node);
    if (d->ref) vsapi->freeNode(d->ref);
    delete d;
}

void VS_CC bm3d_create(const VSMap* in, VSMap* out, void* user, VSCore* core, const VSAPI* vsapi) {
    (void)user;
    auto* d = new Filter();
    int err = 0;
    d->node = vsapi->mapGetNode(in, "clip", 0, nullptr);
    d->vi = vsapi->getVideoInfo(d->node);
    d->ref = vsapi->mapGetNode(in, "ref", 0, &err);
    if (err) d->ref = nullptr;

    vsfeel_bm3d_args args;
    vsfeel_bm3d_args_init(&args);
    read_float_array(vsapi, in, "sigma", args.sigma, &args.sigma_count);
    read_int_array(vsapi, in, "block_step", args.block_step, &args.block_step_count);
    read_int_array(vsapi, in, "bm_range", args.bm_range, &args.bm_range_count);
    read_int(vsapi, in, "radius", &args.radius, &args.radius_set);
    read_int_array(vsapi, in, "ps_num", args.ps_num, &args.ps_num_count);
    read_int_array(vsapi, in, "ps_range", args.ps_range, &args.ps_range_count);
    read_int(vsapi, in, "num_streams", &args.num_streams, &args.num_streams_set);
    read_int(vsapi, in, "extractor_exp", &args.extractor_exp, &args.extractor_exp_set);
    const vsfeel_bm3d_video_info vi = info_of(d->vi);
    vsfeel_bm3d_video_info ref_vi{};
    if (d->ref) {
        ref_vi = info_of(vsapi->getVideoInfo(d->ref));
        args.has_ref = 1;
        args.ref_info = &ref_vi;
    }
    if (vsfeel_bm3d_create(&args, &vi, 0, &d->ctx) != VSFEEL_OK) {
        // the library's message already starts with "BM3D: "
        vsapi->mapSetError(out, vsfeel_bm3d_last_error());
        vsapi->freeNode(d->node);
        if (d->ref) vsapi->freeNode(d->ref);
        delete d;
        return;
    }
    VSFilterDependency deps[2] = {{d->node, rpGeneral}, {d->ref, rpGeneral}};
    vsapi->createVideoFilter(out, "BM3D", d->vi, bm3d_get_frame, bm3d_free, fmParallel, deps,
                             d->ref ? 2 : 1, d, core);
}

}  // namespace

VS_EXTERNAL_API(void) VapourSynthPluginInit2(VSPlugin* plugin, const VSPLUGINAPI* vspapi) {
    vspapi->configPlugin("com.thefeeltrain.vsfeel", "vsfeel",
                         "BM3Dv2 on NVIDIA B200 (CUDA, sm_100a)", VS_MAKE_VERSION(1, 0),
                         VAPOURSYNTH_API_VERSION, 0, plugin);
    // byte-identical to the reference's registration (src/bm3d.cpp:1562-1571)
    vspapi->registerFunction("BM3Dv2",
                             "clip:vnode;"
                             "ref:vnode:opt;"
                             "sigma:float[]:opt;"
                             "block_step:int[]:opt;"
                             "bm_range:int[]:opt;"
                             "radius:int:opt;"
                             "ps_num:int[]:opt;"
                             "ps_range:int[]:opt;"
                             "num_streams:int:opt;"
                             "extractor_exp:int:opt;",
                             "clip:vnode;", bm3d_create, nullptr, plugin);
}
