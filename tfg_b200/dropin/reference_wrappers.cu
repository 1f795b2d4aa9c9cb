// The reference-side binding: the reference's host entry points, written
// against its own unmodified headers, with their bodies replaced by calls into
// libtfgpt's C ABI.  A maintainer who keeps main.cpp links this file (and
// libtfgpt) instead of RenderKernel.cu, NrcKernel.cu, tinybvh_wrapper.cpp and
// mlp.cpp:
//
//   RenderKernel.h:47-77   launchKernelRenderTiny, launchKernelComposite,
//                          launchInicializarCamara, launchKernelCalcularTargets,
//                          launchKernelPrepararInferenciaTail (launchKernelRender,
//                          the reference's own binary-BVH kernel, is not carried)
//   NrcKernel.h:24-41      the four NRC data launchers
//   tinybvh_wrapper.h:22-50 class TinyBVH (the C-ABI hand-off kept in the
//                          class's opaque cwbvh_ptr member)
//   mlp.h:19-44            class ColorMLP (the replacement header beside this file)
//
// Every reference struct is byte-identical to its Tfg* counterpart (checked
// below against the reference's own definitions), so pointers pass through
// unchanged.  The reference's wrappers return void and never check; these
// print the library's error message instead, and run on the legacy default
// stream as the reference's launches did (RenderKernel.cu:270).
//
// The extern "C" functions at the end call the wrappers with the reference's
// own argument types (dim3, TinyBVHD_GPU and ImagenGPU by value) from plain
// pointers, for tests that compare them with the C ABI called directly.
#include <cstddef>
#include <cstdio>
#include <vector>

#include "NrcKernel.h"
#include "RenderKernel.h"
#include "mlp.h"
#include "tfg_pt.h"
#include "tinybvh_wrapper.h"

static_assert(sizeof(Primitiva) == sizeof(TfgPrimitiva), "Primitiva layout");
static_assert(offsetof(Primitiva, triangulo) == offsetof(TfgPrimitiva, u), "Primitiva union offset");
static_assert(offsetof(Primitiva, indice_refraccion) == offsetof(TfgPrimitiva, indice_refraccion), "Primitiva ior");
static_assert(sizeof(LuzPuntual) == sizeof(TfgLuzPuntual), "LuzPuntual layout");
static_assert(sizeof(Camara) == sizeof(TfgCamara), "Camara layout");
static_assert(sizeof(Color) == sizeof(TfgColor), "Color layout");
static_assert(sizeof(DatosMLP) == sizeof(TfgDatosMLP), "DatosMLP layout");
static_assert(sizeof(RegistroEntrenamiento) == sizeof(TfgRegistroEntrenamiento), "RegistroEntrenamiento layout");
static_assert(offsetof(RegistroEntrenamiento, valido) == offsetof(TfgRegistroEntrenamiento, valido), "valido offset");
static_assert(sizeof(SceneBounds) == sizeof(TfgSceneBounds), "SceneBounds layout");
static_assert(sizeof(TinyBVHD_GPU) == sizeof(TfgTinyBVHD_GPU), "TinyBVHD_GPU layout");
static_assert(offsetof(TinyBVHD_GPU, num_nodos) == offsetof(TfgTinyBVHD_GPU, num_nodos), "TinyBVHD_GPU counts");
static_assert(sizeof(ImagenGPU) == sizeof(TfgImagenGPU), "ImagenGPU layout");

template <typename T, typename U>
static T as(U* p) {
    return reinterpret_cast<T>(p);
}

static void report(int rc, const char* what) {
    if (rc) std::fprintf(stderr, "%s: %s\n", what, tfgGetLastErrorString());
}

// ------------------------------------------------------------------ RenderKernel.h
void launchKernelRenderTiny(dim3, dim3, const Camara* camara, const Primitiva* primitivas, int num_primitivas,
                            const LuzPuntual* luces, int num_luces, const Primitiva* primitivas_malla,
                            int num_primitivas_malla, int ancho_img, int alto_img, int samples_per_pixel,
                            int frame_number, TinyBVHD_GPU nodos_bvh, const Primitiva* primitivas_bvh,
                            int num_nodos_bvh, ImagenGPU imagen_directa, unsigned int* dev_counter,
                            RegistroEntrenamiento* buffer_registros, unsigned int* counter_train, int max_cap_train,
                            DatosMLP* buffer_inference, Color* buffer_throughput, bool usar_red_inferencia,
                            bool entrenar_red) {
    const TfgImagenGPU im{imagen_directa.anchura, imagen_directa.altura, as<TfgColor*>(imagen_directa.datos)};
    report(tfgLaunchKernelRenderTiny(as<const TfgCamara*>(camara), as<const TfgPrimitiva*>(primitivas), num_primitivas,
                                     as<const TfgLuzPuntual*>(luces), num_luces,
                                     as<const TfgPrimitiva*>(primitivas_malla), num_primitivas_malla, ancho_img,
                                     alto_img, samples_per_pixel, frame_number,
                                     as<const TfgTinyBVHD_GPU*>(&nodos_bvh), as<const TfgPrimitiva*>(primitivas_bvh),
                                     num_nodos_bvh, &im, dev_counter, as<TfgRegistroEntrenamiento*>(buffer_registros),
                                     counter_train, max_cap_train, as<TfgDatosMLP*>(buffer_inference),
                                     as<TfgColor*>(buffer_throughput), usar_red_inferencia ? 1 : 0,
                                     entrenar_red ? 1 : 0, nullptr),
           "launchKernelRenderTiny");
}

void launchKernelRender(dim3, dim3, const Camara*, const Primitiva*, int, const LuzPuntual*, int, const Primitiva*,
                        int, int, int, int, int, const NodoBVH*, const Primitiva*, int, ImagenGPU, unsigned int*,
                        RegistroEntrenamiento*, unsigned int*, int, DatosMLP*, Color*, bool, bool) {
    std::fprintf(stderr, "launchKernelRender: the binary-BVH kernel is not carried; build a TinyBVH and call "
                         "launchKernelRenderTiny\n");
}

void launchKernelComposite(dim3, dim3, Color* img_pt, Color* img_prediccion, Color* throughput_map, int ancho,
                           int alto) {
    report(tfgLaunchKernelComposite(as<TfgColor*>(img_pt), as<const TfgColor*>(img_prediccion),
                                    as<const TfgColor*>(throughput_map), ancho, alto, nullptr),
           "launchKernelComposite");
}

void launchInicializarCamara(Camara* d_camara, int ancho_imagen, int alto_imagen) {
    report(tfgLaunchInicializarCamara(as<TfgCamara*>(d_camara), ancho_imagen, alto_imagen, nullptr),
           "launchInicializarCamara");
}

void launchKernelCalcularTargets(dim3, dim3, RegistroEntrenamiento* buffer_registros, Color* buffer_prediccion_tail,
                                 DatosMLP* buffer_training_final, int num_elementos) {
    report(tfgLaunchKernelCalcularTargets(as<const TfgRegistroEntrenamiento*>(buffer_registros),
                                          as<const TfgColor*>(buffer_prediccion_tail),
                                          as<TfgDatosMLP*>(buffer_training_final), num_elementos, nullptr),
           "launchKernelCalcularTargets");
}

void launchKernelPrepararInferenciaTail(dim3, dim3, const RegistroEntrenamiento* source_registros,
                                        DatosMLP* dest_inference_inputs, int num_elements) {
    report(tfgLaunchKernelPrepararInferenciaTail(as<const TfgRegistroEntrenamiento*>(source_registros),
                                                 as<TfgDatosMLP*>(dest_inference_inputs), num_elements, nullptr),
           "launchKernelPrepararInferenciaTail");
}

// ------------------------------------------------------------------ NrcKernel.h
void launchGenerarIndicesAleatorios(int, int, cudaStream_t stream, int* indices, int max_range, int count,
                                    unsigned int seed) {
    report(tfgLaunchGenerarIndicesAleatorios(indices, max_range, count, seed, stream),
           "launchGenerarIndicesAleatorios");
}

void launchPrepararDatosEntrenamiento(int, int, cudaStream_t stream, const DatosMLP* buffer,
                                      const int* indices_aleatorios, int batch_size, int n_in, int n_out,
                                      SceneBounds bounds, float* input_matrix, float* target_matrix) {
    report(tfgLaunchPrepararDatosEntrenamiento(as<const TfgDatosMLP*>(buffer), indices_aleatorios, batch_size, n_in,
                                               n_out, as<const TfgSceneBounds*>(&bounds), input_matrix,
                                               target_matrix, stream),
           "launchPrepararDatosEntrenamiento");
}

void launchPrepararDatosInferencia(int, int, cudaStream_t stream, const DatosMLP* datos, uint32_t n_elements,
                                   uint32_t n_in, float* buffer_in, SceneBounds bounds) {
    report(tfgLaunchPrepararDatosInferencia(as<const TfgDatosMLP*>(datos), n_elements, n_in, buffer_in,
                                            as<const TfgSceneBounds*>(&bounds), stream),
           "launchPrepararDatosInferencia");
}

void launchGuardarSalidaInferencia(int, int, cudaStream_t stream, float* network_output, Color* buffer_color,
                                   int n_elements) {
    report(tfgLaunchGuardarSalidaInferencia(network_output, as<TfgColor*>(buffer_color), n_elements, stream),
           "launchGuardarSalidaInferencia");
}

// ------------------------------------------------------------------ tinybvh_wrapper.h
// The C-ABI hand-off lives behind the class's opaque cwbvh_ptr member.
static TfgTinyBVH* handoff(void* p) { return static_cast<TfgTinyBVH*>(p); }

TinyBVH::TinyBVH() : datos_gpu{}, cwbvh_ptr(new TfgTinyBVH{}), primitivas_gpu(nullptr) {}

TinyBVH::~TinyBVH() {
    tfgTinyBVHLiberar(handoff(cwbvh_ptr));
    delete handoff(cwbvh_ptr);
}

void TinyBVH::construirBVH(const std::vector<Primitiva>& primitivas_host) {
    TfgTinyBVH* h = handoff(cwbvh_ptr);
    tfgTinyBVHLiberar(h);
    *h = TfgTinyBVH{};
    report(tfgTinyBVHConstruir(as<const TfgPrimitiva*>(primitivas_host.data()), (int32_t)primitivas_host.size(), h),
           "TinyBVH::construirBVH");
    datos_gpu.d_nodos = as<float4*>(h->ref.d_nodos);
    datos_gpu.d_tris = as<float4*>(h->ref.d_tris);
    datos_gpu.num_nodos = h->ref.num_nodos;
    datos_gpu.num_tris = h->ref.num_tris;
    d_nodos = datos_gpu.d_nodos;
    d_tris = datos_gpu.d_tris;
    primitivas_gpu = as<Primitiva*>(h->d_primitivas);
    num_primitivas_gpu = h->num_primitivas;
}

void TinyBVH::obtenerInfo() {
    std::printf("CWBVH: %u nodes, %u triangles, depth %u\n", datos_gpu.num_nodos, datos_gpu.num_tris,
                handoff(cwbvh_ptr)->max_depth);
}
TinyBVHD_GPU TinyBVH::obtenerDatosGPU() const { return datos_gpu; }
const TinyBVHD_GPU* TinyBVH::getNodosGPU() const { return &datos_gpu; }
const Primitiva* TinyBVH::getPrimitivasGPU() const { return primitivas_gpu; }
unsigned int TinyBVH::getNumNodos() const { return datos_gpu.num_nodos; }
unsigned int TinyBVH::getNumPrimitivas() const { return num_primitivas_gpu; }

// ------------------------------------------------------------------ mlp.h (replacement beside this file)
ColorMLP::ColorMLP(uint32_t n_in, uint32_t n_out, uint32_t batch, const char*) {
    report(tfgMlpCreate(n_in, n_out, batch, 1337, &model_), "ColorMLP");
}
ColorMLP::~ColorMLP() { tfgMlpDestroy(model_); }

float ColorMLP::train_step(DatosMLP* buffer_samples_gpu, uint32_t n_total_samples_disponibles) {
    float loss = 0.0f;
    report(tfgMlpTrainStep(model_, as<const TfgDatosMLP*>(buffer_samples_gpu), n_total_samples_disponibles, &loss,
                           nullptr),
           "ColorMLP::train_step");
    return loss;
}

void ColorMLP::inference(DatosMLP* buffer_samples_gpu, Color* output_gpu, uint32_t n_samples) {
    report(tfgMlpInference(model_, as<const TfgDatosMLP*>(buffer_samples_gpu), as<TfgColor*>(output_gpu), n_samples,
                           nullptr),
           "ColorMLP::inference");
}

void ColorMLP::setBounds(const Vector3d& min, const Vector3d& max) {
    const SceneBounds b{min, max};
    report(tfgMlpSetBounds(model_, as<const TfgSceneBounds*>(&b)), "ColorMLP::setBounds");
}

void ColorMLP::save_model(const std::string& filename) {
    report(tfgMlpSave(model_, filename.c_str()), "ColorMLP::save_model");
}

bool ColorMLP::load_model(const std::string& filename) { return tfgMlpLoad(model_, filename.c_str()) == 0; }

// ------------------------------------------------------------------ test entry points
// The reference's call shapes driven from plain pointers (16 x 16 blocks as
// main.cpp:866-868; the wrappers ignore the launch shape).
extern "C" {

int dropin_render_tiny(const void* camara, const void* prims, int nprims, const void* luces, int nluces, int W, int H,
                       int frame, void* d_nodos, void* d_tris, unsigned num_nodos, unsigned num_tris,
                       const void* bvh_prims, int n_bvh_prims, void* img, void* thr) {
    TinyBVHD_GPU bvh;
    bvh.d_nodos = static_cast<float4*>(d_nodos);
    bvh.d_tris = static_cast<float4*>(d_tris);
    bvh.num_nodos = num_nodos;
    bvh.num_tris = num_tris;
    ImagenGPU im(W, H, static_cast<Color*>(img));
    launchKernelRenderTiny(dim3((W + 15) / 16, (H + 15) / 16), dim3(16, 16), static_cast<const Camara*>(camara),
                           static_cast<const Primitiva*>(prims), nprims, static_cast<const LuzPuntual*>(luces),
                           nluces, nullptr, 0, W, H, 1, frame, bvh, static_cast<const Primitiva*>(bvh_prims),
                           n_bvh_prims, im, nullptr, nullptr, nullptr, 0, nullptr, static_cast<Color*>(thr), false,
                           false);
    return (int)cudaDeviceSynchronize();
}

// TinyBVH built through the class, then a render of its tree through the
// wrapper above; the tree stays alive until dropin_bvh_free.
void* dropin_bvh_build(const void* prims_host, int n, unsigned* num_nodos, unsigned* num_tris,
                       unsigned* num_prims) {
    const Primitiva* p = static_cast<const Primitiva*>(prims_host);
    std::vector<Primitiva> v(p, p + n);
    TinyBVH* b = new TinyBVH();
    b->construirBVH(v);
    *num_nodos = b->getNumNodos();
    *num_tris = b->obtenerDatosGPU().num_tris;
    *num_prims = b->getNumPrimitivas();
    return b;
}

int dropin_bvh_render(void* bvh, const void* camara, const void* prims, int nprims, const void* luces, int nluces,
                      int W, int H, int frame, void* img, void* thr) {
    TinyBVH* b = static_cast<TinyBVH*>(bvh);
    ImagenGPU im(W, H, static_cast<Color*>(img));
    launchKernelRenderTiny(dim3((W + 15) / 16, (H + 15) / 16), dim3(16, 16), static_cast<const Camara*>(camara),
                           static_cast<const Primitiva*>(prims), nprims, static_cast<const LuzPuntual*>(luces),
                           nluces, nullptr, 0, W, H, 1, frame, b->obtenerDatosGPU(), b->getPrimitivasGPU(),
                           (int)b->getNumPrimitivas(), im, nullptr, nullptr, nullptr, 0, nullptr,
                           static_cast<Color*>(thr), false, false);
    return (int)cudaDeviceSynchronize();
}

void dropin_bvh_free(void* bvh) { delete static_cast<TinyBVH*>(bvh); }

// ColorMLP through the replacement class: `steps` train steps on a training
// buffer, then inference of `n` samples; returns the last loss.
float dropin_mlp_train_infer(const void* train_buf, unsigned n_avail, int steps, const double* lo, const double* hi,
                             const void* queries, void* out, unsigned n) {
    ColorMLP m(15, 3, 16384);
    m.setBounds(Vector3d(lo[0], lo[1], lo[2]), Vector3d(hi[0], hi[1], hi[2]));
    float loss = 0.0f;
    for (int k = 0; k < steps; ++k)
        loss = m.train_step(const_cast<DatosMLP*>(static_cast<const DatosMLP*>(train_buf)), n_avail);
    m.inference(const_cast<DatosMLP*>(static_cast<const DatosMLP*>(queries)), static_cast<Color*>(out), n);
    cudaDeviceSynchronize();
    return loss;
}

}  // extern "C"
