"""The reference-side binding (tfg_b200/dropin/reference_wrappers.cu) compiles
against the reference's own, unmodified headers -- RenderKernel.h, NrcKernel.h,
tinybvh_wrapper.h, mlp_types.h -- with the replacement mlp.h beside it, links
to libtfgpt.so, and defines every host entry point of RenderKernel.h:47-77,
NrcKernel.h:24-41, class TinyBVH (tinybvh_wrapper.h:22-50) and class ColorMLP
(mlp.h:19-44) with the reference's C++ signatures.  Its static asserts check
every shared struct against the reference's own definition at compile time."""
import ctypes
import shutil
import subprocess

import pytest

from tfg_b200.dropin import build_dropin

REFERENCE_SYMBOLS = [
    "launchKernelRenderTiny(dim3, dim3, Camara const*, Primitiva const*, int, LuzPuntual const*, int, "
    "Primitiva const*, int, int, int, int, int, TinyBVHD_GPU, Primitiva const*, int, ImagenGPU, unsigned int*, "
    "RegistroEntrenamiento*, unsigned int*, int, DatosMLP*, Color*, bool, bool)",
    "launchKernelComposite(dim3, dim3, Color*, Color*, Color*, int, int)",
    "launchInicializarCamara(Camara*, int, int)",
    "launchKernelCalcularTargets(dim3, dim3, RegistroEntrenamiento*, Color*, DatosMLP*, int)",
    "launchKernelPrepararInferenciaTail(dim3, dim3, RegistroEntrenamiento const*, DatosMLP*, int)",
    "launchGenerarIndicesAleatorios(int, int, CUstream_st*, int*, int, int, unsigned int)",
    "launchPrepararDatosEntrenamiento(int, int, CUstream_st*, DatosMLP const*, int const*, int, int, int, "
    "SceneBounds, float*, float*)",
    "launchPrepararDatosInferencia(int, int, CUstream_st*, DatosMLP const*, unsigned int, unsigned int, float*, "
    "SceneBounds)",
    "launchGuardarSalidaInferencia(int, int, CUstream_st*, float*, Color*, int)",
    "TinyBVH::construirBVH(std::vector<Primitiva, std::allocator<Primitiva> > const&)",
    "TinyBVH::obtenerDatosGPU() const",
    "TinyBVH::getPrimitivasGPU() const",
    "TinyBVH::getNumPrimitivas() const",
    "ColorMLP::train_step(DatosMLP*, unsigned int)",
    "ColorMLP::inference(DatosMLP*, Color*, unsigned int)",
    "ColorMLP::setBounds(Vector3d const&, Vector3d const&)",
]


def test_binding_compiles_against_the_reference_headers(built):
    if build_dropin.reference_dir() is None:
        pytest.skip("reference headers not available (TFG_REFERENCE_DIR)")
    lib = build_dropin.build(force=True)
    assert lib is not None and lib.exists()
    nm = shutil.which("nm")
    if nm:
        out = subprocess.run([nm, "-DC", "--defined-only", str(lib)], capture_output=True, text=True).stdout
        missing = [s for s in REFERENCE_SYMBOLS if s not in out]
        assert not missing, f"reference entry points not defined: {missing}"
    # loads without a GPU against the library it was linked to
    dl = ctypes.CDLL(str(lib))
    for name in ("dropin_render_tiny", "dropin_bvh_build", "dropin_bvh_render", "dropin_bvh_free",
                 "dropin_mlp_train_infer"):
        assert hasattr(dl, name)
