// ORACLE -- test infrastructure only.  Compiles the reference's own host/shader shared headers
// (src/Shaders/compat/*.h of Stratum2, with its vendored Eigen) and exposes their packing code,
// so tests can pin this project's byte layouts against the reference itself.  Built by
// oracle/build_oracle.py into oracle/_ref/ when the reference tree is available.
#include <Core/math.hpp>

namespace stm2 { class Node; }

#include <Shaders/compat/common.h>
#include <Shaders/compat/material_data.h>
#include <Shaders/compat/scene.h>
#include <Shaders/compat/transform.h>

using namespace stm2;

extern "C" {

// PackedMaterialData setters (material_data.h:51-73) as used by makeMetallicRoughnessMaterial
// (src/App/Scene.cpp:195-208) or with explicit Disney parameters.
// params: baseColor rgb, emission rgb, specular, sheen, metallic, roughness, anisotropic,
//         subsurface, clearcoat, clearcoatGloss, transmission, etaMinus1  (18 floats)
void ref_pack_material(const float* p, uint32_t* words_out, float* emission_scale_out) {
    PackedMaterialData m;
    m.mPackedData = uint4::Zero();
    m.mEmissionScale = 0;
    m.setBaseColor(float3(p[0], p[1], p[2]));
    m.setEmission(float3(p[3], p[4], p[5]));
    m.setSpecular(p[6]);
    m.setSheen(p[7]);
    m.setMetallic(p[8]);
    m.setRoughness(p[9]);
    m.setAnisotropic(p[10]);
    m.setSubsurface(p[11]);
    m.setClearcoat(p[12]);
    m.setClearcoatGloss(p[13]);
    m.setTransmission(p[14]);
    m.setEta(p[15]);
    for (int i = 0; i < 4; ++i) words_out[i] = m.mPackedData[i];
    *emission_scale_out = m.mEmissionScale;
}

// PackedMaterialData getters: baseColor rgb, emission rgb, specular, sheen, metallic, roughness,
// anisotropic, subsurface, clearcoat, clearcoatGloss, transmission, eta (16 floats)
void ref_unpack_material(const uint32_t* words, float emission_scale, float* out) {
    PackedMaterialData m;
    for (int i = 0; i < 4; ++i) m.mPackedData[i] = words[i];
    m.mEmissionScale = emission_scale;
    const float3 b = m.getBaseColor(), e = m.getEmission();
    out[0] = b[0]; out[1] = b[1]; out[2] = b[2];
    out[3] = e[0]; out[4] = e[1]; out[5] = e[2];
    out[6] = m.getSpecular(); out[7] = m.getSheen(); out[8] = m.getMetallic(); out[9] = m.getRoughness();
    out[10] = m.getAnisotropic(); out[11] = m.getSubsurface(); out[12] = m.getClearcoat();
    out[13] = m.getClearcoatGloss(); out[14] = m.getTransmission(); out[15] = m.getEta();
}

// MeshInstanceData (scene.h:46-58): 2 words
void ref_mesh_instance(uint32_t material_address, uint32_t vertex_info_index, uint32_t primitive_count, uint32_t* out) {
    MeshInstanceData d(material_address, vertex_info_index, primitive_count);
    out[0] = d.mTypeMaterialAddress;
    out[1] = d.mData;
}

// MeshVertexInfo (scene.h:89-132): 8 words
void ref_vertex_info(const uint32_t* a, uint32_t* out) {
    MeshVertexInfo v(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8], a[9], a[10], a[11]);
    static_assert(sizeof(MeshVertexInfo) == 32, "MeshVertexInfo is 32 bytes");
    std::memcpy(out, &v, 32);
}

// ProjectionData::makePerspective (transform.h:181-190): 8 floats
void ref_make_perspective(float fovy, float aspect, float znear, float* out) {
    ProjectionData p = ProjectionData::makePerspective(fovy, aspect, float2(0, 0), znear);
    out[0] = p.mScale[0]; out[1] = p.mScale[1]; out[2] = p.mOffset[0]; out[3] = p.mOffset[1];
    out[4] = p.mNearPlane; out[5] = p.mFarPlane; out[6] = p.mSensorArea; out[7] = p.mVerticalFoV;
}

// ProjectionData::backProject (transform.h:159-170)
void ref_back_project(const float* proj, float cx, float cy, float* out) {
    ProjectionData p;
    p.mScale = float2(proj[0], proj[1]); p.mOffset = float2(proj[2], proj[3]);
    p.mNearPlane = proj[4]; p.mFarPlane = proj[5]; p.mSensorArea = proj[6]; p.mVerticalFoV = proj[7];
    const float3 r = p.backProject(float2(cx, cy));
    out[0] = r[0]; out[1] = r[1]; out[2] = r[2];
}

// colour helpers of compat/common.h (51, 88-104): rgbToSrgb, viridisQuintic, luminance
void ref_rgb_to_srgb(const float* rgb, float* out) {
    const float3 r = rgbToSrgb(float3(rgb[0], rgb[1], rgb[2]));
    out[0] = r[0]; out[1] = r[1]; out[2] = r[2];
}
void ref_viridis(float x, float* out) {
    const float3 r = viridisQuintic(x);
    out[0] = r[0]; out[1] = r[1]; out[2] = r[2];
}
float ref_luminance(const float* rgb) { return luminance(float3(rgb[0], rgb[1], rgb[2])); }

// sizes of the shared structs
void ref_sizes(uint32_t* out) {
    out[0] = sizeof(InstanceData);
    out[1] = sizeof(MeshVertexInfo);
    out[2] = sizeof(TransformData);
    out[3] = sizeof(ProjectionData);
    out[4] = sizeof(ViewData);
    out[5] = sizeof(ShadingData);
    out[6] = sizeof(PackedMaterialData);
}

}  // extern "C"
