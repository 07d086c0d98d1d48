/*
 * sheen_types.h -- byte layout of every array a Sheen scene is made of.
 *
 * This is the binary contract between a caller (the Blender add-on, the
 * native Python module, the CLI) and the renderer core.  Every struct here
 * has the same size, alignment and field offsets as its counterpart in the
 * reference's types.h (types.h:24-301); the field names are kept too, because
 * ctypes callers address fields by name.  The header is plain C (C99 with a
 * GNU alignment attribute) so that it can be included from C, C++ and CUDA
 * without the CUDA runtime headers: a float3 here is three packed floats,
 * 12 bytes with 4-byte alignment, exactly like CUDA's float3.
 *
 * Sizes (checked by static asserts in sheen_b200/csrc/abi_check.cpp and by
 * tests/test_abi.py):
 *   Ray 32, HitRecord 80, CameraData 64, Material 112, Triangle 112,
 *   TextureRef 16(+pad), Object 48, Light 96, Medium 48, Plane 32,
 *   SweepPoint 16, SweepStrand 16, HeightField 64, LathePoint 16, Lathe 32,
 *   PrismPoint 16, Prism 48, CSGNode 32, Superellipsoid 48, SheenScene 352.
 */
#ifndef SHEEN_TYPES_H
#define SHEEN_TYPES_H

#define SHEEN_ALIGN16 __attribute__((aligned(16)))

/* Same size and alignment as CUDA's float3 (12 B, 4-aligned) and float2 (8 B, 8-aligned). */
typedef struct sheen_float3 { float x, y, z; } sheen_float3;
typedef struct __attribute__((aligned(8))) sheen_float2 { float x, y; } sheen_float2;

#ifdef __cplusplus
extern "C" {
#endif

/* types.h:24-29 */
typedef struct SHEEN_ALIGN16 SheenRay {
    sheen_float3 origin;
    sheen_float3 direction;
    float t_min;
    float t_max;
} SheenRay;

/* types.h:49-58.  focal_length == 0 selects the legacy camera where the
 * length of `forward` sets the field of view. */
typedef struct SHEEN_ALIGN16 CameraData {
    sheen_float3 position;
    sheen_float3 right;
    sheen_float3 up;
    sheen_float3 forward;
    float focal_length;   /* mm */
    float sensor_width;   /* mm */
    float shift_x;
    float shift_y;
} CameraData;

/* types.h:63-85 */
typedef struct SHEEN_ALIGN16 Material {
    sheen_float3 diffuse_color;
    float specular;
    float shininess;        /* < 0: shadow debug colour mode */
    float ambient;
    int   texture_id;       /* -1: none */
    int   _pad_tex;
    float anisotropy;       /* > 0: strand (hair) lobe model */
    float hair_shift;
    float hair_spec_r;
    float hair_exp_r;
    float hair_spec_t;
    float hair_exp_t;
    float hair_backlight;
    float reflect;          /* mirror weight of the single reflection bounce */
    float transmission;     /* > 0: refractive */
    float ior;
    sheen_float3 emission_color;
    float emission;
    int   mask_id;          /* property map: R transmission, G ior-1, B roughness */
    int   normal_id;        /* tangent-space normal map */
    float normal_strength;
} Material;

/* types.h:90-96 */
typedef struct SHEEN_ALIGN16 Triangle {
    sheen_float3 v0, v1, v2;
    sheen_float3 n0, n1, n2;  /* all zero: flat shading */
    sheen_float2 uv0, uv1, uv2;
    int material_id;
    int _pad0, _pad1;
} Triangle;

/* types.h:100-105 -- device-side view of one texture's mip chain */
typedef struct SHEEN_ALIGN16 TextureRef {
    const unsigned char* pixels;
    int width;
    int height;
    int mips;
} TextureRef;

/* types.h:110-116 -- spheres (type 0) */
typedef struct SHEEN_ALIGN16 Object {
    int type;
    int material_id;
    sheen_float3 param1;    /* centre */
    float param2;           /* radius */
    float _pad0, _pad1, _pad2;
} Object;

/* types.h:130-145.  type 0 sun, 1 point, 2 area, 3 spot; flags bit0 = lights media */
typedef struct SHEEN_ALIGN16 Light {
    sheen_float3 direction;
    sheen_float3 position;
    sheen_float3 u_axis;
    sheen_float3 v_axis;
    sheen_float3 color;
    float intensity;
    float radius;
    float angle;
    float blend;
    float beam;
    int   type;
    int   flags;
    int   texture_id;
    int   _pad1;
} Light;

/* types.h:152-159 */
typedef struct SHEEN_ALIGN16 Medium {
    sheen_float3 center;
    sheen_float3 half;
    sheen_float3 sigma_s;
    float sigma_t;
    int   samples;
    int   _pad0;
} Medium;

/* types.h:164-169 -- dot(p, normal) + d = 0 */
typedef struct SHEEN_ALIGN16 Plane {
    sheen_float3 normal;
    float d;
    int material_id;
    int _pad0, _pad1, _pad2;
} Plane;

/* types.h:174-187 */
typedef struct SHEEN_ALIGN16 SweepPoint {
    sheen_float3 position;
    float radius;
} SweepPoint;

typedef struct SHEEN_ALIGN16 SweepStrand {
    int point_offset;
    int point_count;
    int material_id;
    int _pad0;
} SweepStrand;

/* types.h:201-217.  image != NULL selects the 8-bit height map mode. */
typedef struct SHEEN_ALIGN16 HeightField {
    sheen_float3 center;
    float size_x;
    float size_z;
    float height;
    float freq;
    int   octaves;
    int   seed;
    int   material_id;
    const unsigned char* image;
    int   img_w;
    int   img_h;
    int   _pad0;
} HeightField;

/* types.h:225-237 */
typedef struct SHEEN_ALIGN16 LathePoint {
    float y;
    float radius;
    int _pad0, _pad1;
} LathePoint;

typedef struct SHEEN_ALIGN16 Lathe {
    sheen_float3 center;    /* bounds use it; intersection does not (reference behaviour) */
    int point_offset;
    int point_count;
    int material_id;
    int _pad0;
} Lathe;

/* types.h:245-260 */
typedef struct SHEEN_ALIGN16 PrismPoint {
    float x;
    float z;
    int _pad0, _pad1;
} PrismPoint;

typedef struct SHEEN_ALIGN16 Prism {
    sheen_float3 center;
    float y_min;
    float y_max;
    float sweep;
    int point_offset;
    int point_count;
    int material_id;
    int _pad0;
} Prism;

/* types.h:281-287.  leaf_kind -1: interior node, op 0 union / 1 intersection / 2 difference;
 * leaf_kind 0 sphere (objects[]), 1 superellipsoid. */
typedef struct SHEEN_ALIGN16 CSGNode {
    int op;
    int leaf_kind;
    int leaf_index;
    int left;
    int right;
} CSGNode;

/* types.h:293-301 -- |x/a|^n + |y/b|^n + |z/c|^n = 1 */
typedef struct SHEEN_ALIGN16 Superellipsoid {
    sheen_float3 center;
    float a, b, c;
    float n;
    int material_id;
    int _pad0, _pad1;
} Superellipsoid;

#ifdef __cplusplus
}
#endif

#endif /* SHEEN_TYPES_H */
