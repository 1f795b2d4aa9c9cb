// Drop-in replacement for the reference's mlp.h (mlp.h:19-70): the same
// ColorMLP class and public methods over libtfgpt's cache model instead of
// tiny-cuda-nn.  The tiny-cuda-nn JSON configuration argument becomes an
// optional string the model ignores: the network, encoding, loss and
// optimiser are fixed (the reference's mlp.cpp:22-73 values).  Compile the
// reference's .cpp files with this directory ahead of the reference's own on
// the include path.
#pragma once

#include <cstdint>
#include <string>

#include "mlp_types.h"
#include "tfg_pt.h"

class ColorMLP {
public:
    ColorMLP(uint32_t n_in, uint32_t n_out, uint32_t batch, const char* config_override = nullptr);
    ~ColorMLP();
    ColorMLP(const ColorMLP&) = delete;
    ColorMLP& operator=(const ColorMLP&) = delete;

    // One Adam step on `batch` samples drawn from the buffer; returns the loss
    // (mlp.cpp:95-125, which also synchronised to read it).
    float train_step(DatosMLP* buffer_samples_gpu, uint32_t n_total_samples_disponibles);
    // Scrubbed predictions of n samples into output_gpu (mlp.cpp:127-170).
    void inference(DatosMLP* buffer_samples_gpu, Color* output_gpu, uint32_t n_samples);
    void setBounds(const Vector3d& min, const Vector3d& max);
    void save_model(const std::string& filename);
    bool load_model(const std::string& filename);

    // The underlying C-ABI model (for the calls the reference class lacks).
    TfgColorMLP* handle() const { return model_; }

private:
    TfgColorMLP* model_ = nullptr;
};
