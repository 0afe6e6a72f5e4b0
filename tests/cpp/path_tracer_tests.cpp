// path_tracer_tests.cpp - the reference's GPU integration test
// (tests/path_tracer_tests.cpp of hdCodex) driven through the drop-in
// hdcodex::CudaPathTracer: same scenes, same calls, same checks.
//
// Built by tests/test_cpp_shim.py. Exit code 0: all checks passed;
// 2: no sm_100 device (the constructor threw); 1: a check failed.
#include "hdcx/cuda_path_tracer.h"

#include <array>
#include <cmath>
#include <cstdio>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

void Check(bool condition, const char* message)
{
    if (!condition) throw std::runtime_error(message);
}

std::shared_ptr<hdcodex::SceneSnapshot> BaseScene()
{
    auto scene = std::make_shared<hdcodex::SceneSnapshot>();
    scene->revision = 1;
    hdcodex::SceneMesh mesh;
    mesh.id = "/triangle";
    mesh.positions = {-1.25F, -1.0F, -3.0F, 1.25F, -1.0F, -3.0F, 0.0F, 1.2F, -3.0F};
    mesh.indices = {0, 1, 2};
    mesh.texcoords = {0.0F, 0.0F, 1.0F, 0.0F, 0.5F, 1.0F};
    mesh.materialId = "/red";
    scene->meshes.push_back(mesh);
    hdcodex::SceneMaterial red;
    red.id = "/red";
    red.baseColor = {1.0F, 1.0F, 1.0F};
    red.metalness = 0.15F;
    red.roughness = 0.3F;
    red.baseColorTexture = "green#srgb";
    scene->materials.push_back(red);
    hdcodex::SceneTexture green;
    green.id = "green#srgb";
    green.width = 1;
    green.height = 1;
    green.srgb = true;
    green.rgba = {16, 220, 32, 255};
    scene->textures.push_back(green);
    hdcodex::SceneTexture rect;
    rect.id = "rect#hdr";
    rect.width = 1;
    rect.height = 1;
    rect.rgbaFloat = {2.0F, 2.0F, 2.0F, 1.0F};
    scene->textures.push_back(rect);
    hdcodex::SceneLight dome;
    dome.id = "/dome";
    dome.type = hdcodex::SceneLightType::Dome;
    dome.color = {0.08F, 0.16F, 0.8F};
    dome.intensity = 0.35F;
    scene->lights.push_back(dome);
    hdcodex::SceneLight rectLight;
    rectLight.id = "/rect";
    rectLight.type = hdcodex::SceneLightType::Rect;
    rectLight.color = {1.0F, 0.92F, 0.82F};
    rectLight.intensity = 50.0F;
    rectLight.texture = "rect#hdr";
    rectLight.basisX = {0.817F, -0.576F, 0.0F};
    rectLight.basisY = {0.184F, 0.261F, -0.947F};
    rectLight.basisZ = {0.547F, 0.775F, 0.319F};
    rectLight.position = {3.282F, 4.650F, -1.086F};
    rectLight.axisU = {1.634F, -1.152F, 0.0F};
    rectLight.axisV = {0.368F, 0.522F, -1.894F};
    rectLight.width = 2.0F;
    rectLight.height = 2.0F;
    rectLight.area = 4.0F;
    scene->lights.push_back(rectLight);
    return scene;
}

}  // namespace

int main()
{
    std::unique_ptr<hdcodex::CudaPathTracer> tracerPtr;
    try {
        tracerPtr = std::make_unique<hdcodex::CudaPathTracer>(0);
    } catch (const std::exception& e) {
        std::printf("no CUDA path tracer: %s\n", e.what());
        return 2;
    }
    try {
        hdcodex::CudaPathTracer& tracer = *tracerPtr;
        Check(tracer.GetShadingMode() == hdcodex::ShadingMode::Fused, "fused shading mode is not the default");
        tracer.SetShadingMode(hdcodex::ShadingMode::Modular);
        Check(tracer.GetShadingMode() == hdcodex::ShadingMode::Modular, "modular shading mode not selected");
        tracer.SetShadingMode(hdcodex::ShadingMode::Fused);
        bool rejected = false;
        try {
            tracer.SetShadingMode(hdcodex::ShadingMode::RasterPreview);
        } catch (const std::invalid_argument&) {
            rejected = true;
        }
        Check(rejected, "raster preview was not rejected");
        Check(!tracer.HasGeometry(), "geometry before SetScene");
        hdcodex::PathTracerCamera camera;
        camera.origin = {0.0F, 0.0F, 0.0F};
        camera.lowerLeft = {-1.0F, -1.0F, -1.0F};
        camera.horizontal = {2.0F, 0.0F, 0.0F};
        camera.vertical = {0.0F, 2.0F, 0.0F};
        Check(tracer.Render(camera, 64, 64, 0).empty(), "render without geometry returned pixels");

        auto scene = BaseScene();
        tracer.SetScene(std::shared_ptr<const hdcodex::SceneSnapshot>(scene));
        Check(tracer.HasGeometry(), "path tracer did not build geometry");
        constexpr std::uint32_t width = 64, height = 64;
        const auto sequentialFirst = tracer.Render(camera, width, height, 0U);
        const auto sequentialTwo = tracer.Render(camera, width, height, 1U);
        const auto batchedTwo = tracer.Render(camera, width, height, 0U, 8U, 2U);
        Check(batchedTwo.size() == sequentialTwo.size(), "batched image size changed");
        for (std::size_t i = 0; i < batchedTwo.size(); ++i) {
            Check(std::abs(batchedTwo[i] - sequentialTwo[i]) < 1e-5F, "batched samples changed the progressive estimator");
        }
        Check(sequentialFirst.size() == batchedTwo.size(), "single-sample image size changed");
        const auto pixels = tracer.Render(camera, width, height, 0U, 8U, 64U);
        Check(pixels.size() == width * height * 4U, "wrong image size");
        for (float v : pixels) Check(std::isfinite(v), "non-finite output");
        const std::size_t center = (height / 2U * width + width / 2U) * 4U;
        const float centerLuma = pixels[center] + pixels[center + 1] + pixels[center + 2];
        const float cornerLuma = pixels[0] + pixels[1] + pixels[2];
        Check(std::abs(centerLuma - cornerLuma) > 0.02F, "image does not distinguish triangle from background");
        Check(pixels[center + 1] > pixels[center] * 1.5F, "base-color texture not sampled");
        Check(pixels[center + 3] == 1.0F, "alpha is not one");
        const auto interactive = tracer.Render(camera, width / 2U, height / 2U, 0U, 2U);
        Check(interactive.size() == width * height, "interactive render size");
        tracer.SetScene(std::shared_ptr<const hdcodex::SceneSnapshot>());
        Check(!tracer.HasGeometry(), "SetScene(nullptr) kept geometry");
        std::printf("CudaPathTracer drop-in test passed\n");
        return 0;
    } catch (const std::exception& e) {
        std::printf("FAILED: %s\n", e.what());
        return 1;
    }
}
