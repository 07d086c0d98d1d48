// owned_scene.h -- host-side storage behind SheenOwnedScene: the .sheen
// loader and the synthetic generators fill one, sheen_owned_view() exposes it
// as a SheenScene whose pointers point into these vectors.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "sheen_c_api.h"

namespace sheen {

struct Texture {
    int w = 0, h = 0;
    std::vector<uint8_t> rgb;   // w*h*3, level 0 only (mips are built at upload)
};

struct OwnedScene {
    CameraData camera{};
    std::vector<Object> objects;
    std::vector<SweepPoint> sweep_points;
    std::vector<SweepStrand> sweep_strands;
    std::vector<Triangle> triangles;
    std::vector<HeightField> heightfields;
    std::vector<std::vector<uint8_t>> height_images;   // owned HF image pixels
    std::vector<int> height_image_of;                  // hf index -> image index or -1
    std::vector<Superellipsoid> superellipsoids;
    std::vector<LathePoint> lathe_points;
    std::vector<Lathe> lathes;
    std::vector<PrismPoint> prism_points;
    std::vector<Prism> prisms;
    std::vector<CSGNode> csg_nodes;
    int csg_root = -1;
    std::vector<Plane> planes;
    std::vector<Material> materials;
    std::vector<Texture> textures;
    std::vector<Light> lights;
    std::vector<Medium> media;
    SheenSceneSettings settings{};

    // Scene extensions (SheenSceneExt; the extended generators fill them).
    std::vector<SheenBezierRun> lathe_bezier, prism_bezier;
    std::vector<float> bezier_ctrl;          // (a, b) pairs
    std::vector<float> se_n2;
    std::vector<SheenHeightGrid> hf_grid;
    std::vector<float> hf_heights;
    std::vector<int> csg_roots;
    std::vector<SheenCsgBox> csg_boxes;
    std::vector<SheenCsgCone> csg_cones;
    int max_depth = 0;                       // reflect + refract recursion (SheenSceneExt.max_depth)
    std::vector<Triangle> mesh_triangles;    // instanced meshes (object space)
    std::vector<SheenMesh> meshes;
    std::vector<SheenInstance> instances;

    // C views (rebuilt by finalize()).
    SheenScene view{};
    SheenSceneExt ext_view{};
    std::vector<const unsigned char*> tex_ptrs;
    std::vector<int> tex_w, tex_h;

    OwnedScene();
    void finalize();

    // Builders with the defaults of the reference's Scene::add_* (scene.h:55-408).
    int add_material(float r, float g, float b, float spec, float shin, float amb);
    void add_sphere(float x, float y, float z, float rad, int mat);
    void add_plane(float nx, float ny, float nz, float d, int mat);
    void add_triangle(const float v[9], const float n[9], const float uv[6], int mat);
    void add_point_light(float x, float y, float z, float r, float g, float b, float power, float radius);
    void add_spot_light(const float pos[3], const float dir[3], const float col[3], float power,
                        float half_angle, float blend, float radius, float beam);
    void add_sweep_smooth(const std::vector<SweepPoint>& ctrl, int mat, int subdivs);
    void add_sweep(const std::vector<SweepPoint>& pts, int mat);
    static Light default_light();
};

}  // namespace sheen
