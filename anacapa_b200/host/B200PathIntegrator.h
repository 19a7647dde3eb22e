// B200PathIntegrator — drop-in IIntegrator for the reference renderer
// (include/anacapa/integrator/IIntegrator.h:172-198) that renders whole frames
// on a B200 through the C ABI of include/anacapa_b200.h.
//
// It is compiled inside the reference tree (its include paths: include/ and
// src/), next to PathIntegrator; RenderSession::render selects it in place of
// `std::make_unique<PathIntegrator>(maxDepth)` (src/render/RenderSession.cpp:
// 458-464). `prepare` flattens the SceneView — GeometryPool meshes, the
// CurveBrute's CurvePool, the materials by meshID, the lights, the dome and
// the camera — and uploads it; `renderFrame` renders [sampleStart,
// sampleStart + sampleCount) samples per pixel and merges the result into the
// Film as one full-frame TileBuffer (Film::mergeTile), returning true.
// There is no CPU fallback: unsupported scene content (image textures, a
// rotated dome) makes
// prepare/renderFrame fail with a message in lastError(); renderTile throws.
#pragma once

#include <anacapa/film/Film.h>
#include <anacapa/integrator/IIntegrator.h>

#include <cstdint>
#include <string>

#include "anacapa_b200.h"

namespace anacapa_b200 {

class B200PathIntegrator : public anacapa::IIntegrator {
public:
    // PathIntegrator(maxDepth, minDepth) (src/integrator/PathIntegrator.h:24-25)
    explicit B200PathIntegrator(uint32_t maxDepth = 8, uint32_t minDepth = 2, int device = 0);
    ~B200PathIntegrator() override;
    B200PathIntegrator(const B200PathIntegrator&) = delete;
    B200PathIntegrator& operator=(const B200PathIntegrator&) = delete;

    // A CUDA device was found and a context created (CudaPathIntegrator::isValid).
    bool isValid() const { return m_ctx != nullptr; }
    const std::string& lastError() const { return m_err; }

    void prepare(const anacapa::SceneView& scene) override;

    // Tiles are not rendered on the GPU path (the reference calls renderTile
    // only for adaptive passes); throws std::runtime_error.
    void renderTile(const anacapa::SceneView& scene, const anacapa::TileRequest& tile, uint32_t filmWidth,
                    uint32_t filmHeight, anacapa::ISampler& sampler, anacapa::TileBuffer& localTile) override;

    bool renderFrame(const anacapa::SceneView& scene, uint32_t filmWidth, uint32_t filmHeight,
                     uint32_t sampleStart, uint32_t sampleCount, anacapa::Film& film) override;

    // Statistics of the last frame (rays traced, device time).
    ana_stats stats() const;

    // The host half of prepare, usable without a device: flattens the
    // SceneView for a filmWidth x filmHeight frame and builds the device
    // layout (ana_prepare_scene). Returns null with a message in `err` for
    // unsupported content; the caller frees the result (ana_prepared_free).
    static ana_prepared* prepareHost(const anacapa::SceneView& scene, uint32_t filmWidth, uint32_t filmHeight,
                                     std::string& err);

private:
    bool upload(const anacapa::SceneView& scene);
    bool fail(const std::string& what);

    ana_ctx* m_ctx = nullptr;
    const anacapa::SceneView* m_prepared = nullptr;
    uint32_t m_maxDepth = 8;
    uint32_t m_minDepth = 2;
    std::string m_err;
};

}  // namespace anacapa_b200
