// oracle/_ref driver: the reference's OWN kernel code, compiled as host C++.
//
// TEST INFRASTRUCTURE ONLY. This file is the checker's harness: it instantiates the
// reference's scene templates exactly as its Rust codegen would, and restates the
// 20-line `render` kernel (kernel/ocl/render/render.cl:6-27) because that file uses
// OpenCL vector literals that do not parse as C++. Nothing in the product links it.
//
// What is instantiated (the two scene recipes the CUDA path serves):
//   hyperbolic  SceneImpl<Hyperbolic3, Mapped<PointView, Moebius>,
//                 Vec<Mapped<Covered<Choice{Plane,Horosphere},
//                   Mixture{diffuse: Colored<Lambertian>, specular: Specular,
//                           luminous: Emissive<Absorbing>}>, Moebius>>, ConstBg, H>
//               (main/examples/hearth.rs:27-41,66-105)
//   euclidean   the same with Euclidean3, Homogenous3 maps and Choice{Plane,Sphere}
//               (main/examples/eu.rs:30-44,71 for the Homogenous3 view/object maps)
// The generated-struct text and getter names follow type-macros/src/source.rs:14-92,190
// (struct + `__gc` getters), :171-178 (enum = {usize index; union{..}}) and the
// template-instantiation pattern of types/src/source.rs:134-144 (`#define $Key value`
// + `#include <x.inl>`), as the reference's own fixtures do in
// kernel/ocl/render/test/scene_hy.cpp:1-48.
//
// Input is the serialized scene byte buffer (types/src/io.rs write_entity layout, the
// same bytes the device kernel reads); this file parses it into the host structs
// (host vec<T,3> is 12 bytes, the serialized float3 is 16).

#include <cstdint>
#include <cstring>
#include <cstdlib>
#include <vector>
#include <thread>
#include <mutex>
#include <atomic>

#include <types.hh>
#include <algebra/real.hh>
#include <algebra/vector.hh>
#include <algebra/color.hh>
#include <random.hh>
#include <hash.hh>
#include <render/context.hh>
#include <geometry/hyperbolic.hh>
#include <geometry/euclidean.hh>
#include <geometry/ray_hy.hh>
#include <geometry/ray_eu.hh>
#include <render/light/hy.hh>
#include <render/light/eu.hh>
#include <shape/hy/plane.hh>
#include <shape/hy/horosphere.hh>
#include <shape/eu/plane.hh>
#include <shape/eu/sphere.hh>
#include <material/lambertian.hh>
#include <material/specular.hh>
#include <material/absorbing.hh>
#include <view/point/hy.hh>
#include <view/point/eu.hh>
#include <background/constant.hh>
#include <transform/homogenous.hh>
#include <shape/choice/macros.hh>
#include <material/mixture/macros.hh>

// ---------------------------------------------------------------- light hops (const H)
static uint g_light_hops = 1;

// ---------------------------------------------------------------- per-thread counters
struct RefStats {
    uint64_t samples, hops, object_tests, hits;
};
static thread_local RefStats t_stats;

// ============================================================================ shared
// Material: Mixture{ diffuse: Colored<Lambertian>, specular: Specular,
//                    luminous: Emissive<Absorbing> }  (objects/src/material/mixture.rs)

typedef struct ColoredLambertian { color3 color; } ColoredLambertian;
inline __global const Lambertian *colored_lambertian__inner__gc(__global const ColoredLambertian *) { return NULL; }
#define $Self ColoredLambertian
#define $self colored_lambertian
#define $Material Lambertian
#define $material lambertian
#include <material/colored.inl>
#undef $Self
#undef $self
#undef $Material
#undef $material

typedef struct EmissiveAbsorbing { color3 emission; } EmissiveAbsorbing;
inline __global const Absorbing *emissive_absorbing__inner__gc(__global const EmissiveAbsorbing *) { return NULL; }
#define $Self EmissiveAbsorbing
#define $self emissive_absorbing
#define $Material Absorbing
#define $material absorbing
#include <material/emissive.inl>
#undef $Self
#undef $self
#undef $Material
#undef $material

typedef struct ComponentColoredLambertian { ColoredLambertian material; real portion; } ComponentColoredLambertian;
inline __global const ColoredLambertian *component_colored_lambertian__material__gc(__global const ComponentColoredLambertian *s) { return &s->material; }
typedef struct ComponentSpecular { real portion; } ComponentSpecular;
inline __global const Specular *component_specular__material__gc(__global const ComponentSpecular *) { return NULL; }
typedef struct ComponentEmissiveAbsorbing { EmissiveAbsorbing material; real portion; } ComponentEmissiveAbsorbing;
inline __global const EmissiveAbsorbing *component_emissive_absorbing__material__gc(__global const ComponentEmissiveAbsorbing *s) { return &s->material; }

typedef struct HtMixture {
    ComponentColoredLambertian diffuse;
    ComponentSpecular specular;
    ComponentEmissiveAbsorbing luminous;
} HtMixture;
#define $Self HtMixture
#define $self ht_mixture
#define $mixture_interact_list \
    mixture_interact_component(colored_lambertian, component_colored_lambertian, diffuse) \
    mixture_interact_component(specular, component_specular, specular) \
    mixture_interact_component(emissive_absorbing, component_emissive_absorbing, luminous)
#include <material/mixture/impl.inl>
#undef $Self
#undef $self
#undef $mixture_interact_list

// ============================================================================ hyperbolic
// Shape: Choice { Plane(Plane), Horosphere(Horosphere) }  (zero-sized variants)
typedef struct HtHyChoice { usize index; } HtHyChoice;
inline __global const void *ht_hy_choice__Plane__gc(__global const HtHyChoice *) { return NULL; }
inline __global const Plane *ht_hy_choice__Plane__field_0__gc(__global const void *) { return NULL; }
inline __global const void *ht_hy_choice__Horosphere__gc(__global const HtHyChoice *) { return NULL; }
inline __global const Horosphere *ht_hy_choice__Horosphere__field_0__gc(__global const void *) { return NULL; }
typedef HtHyChoice ShapeHtHyChoice;
#define $Self ShapeHtHyChoice
#define $self shape_ht_hy_choice
#define $Geo Hy
#define $geo hy
#define $shape_choice_detect_list \
    shape_choice_detect_variant(ht_hy_choice, 0, plane_hy, Plane) \
    shape_choice_detect_variant(ht_hy_choice, 1, horosphere, Horosphere)
#include <shape/choice/impl.inl>
#undef $Self
#undef $self
#undef $Geo
#undef $geo
#undef $shape_choice_detect_list

// Object: Covered<Hy, Choice, Mixture>
typedef struct HtHyCovered { HtMixture material; HtHyChoice shape; } HtHyCovered;
typedef struct HtHyCoveredCache { HyDir normal; } HtHyCoveredCache;
inline __global const ShapeHtHyChoice *ht_hy_covered__shape__gc(__global const HtHyCovered *s) { return &s->shape; }
inline __global const HtMixture *ht_hy_covered__material__gc(__global const HtHyCovered *s) { return &s->material; }
#define $Self HtHyCovered
#define $self ht_hy_covered
#define $Geo Hy
#define $geo hy
#define $Shape ShapeHtHyChoice
#define $shape shape_ht_hy_choice
#define $Material HtMixture
#define $material ht_mixture
#define $Cache HtHyCoveredCache
#define $cache ht_hy_covered_cache
#include <object/covered.inl>
#undef $Self
#undef $self
#undef $Geo
#undef $geo
#undef $Shape
#undef $shape
#undef $Material
#undef $material
#undef $Cache
#undef $cache

// RayMap<Hy, Moebius> -> ray_hy_map_mo
#define $Geo Hy
#define $geo hy
#define $Map Moebius
#define $map mo
#include <geometry/ray_map.inl>
#undef $Geo
#undef $geo
#undef $Map
#undef $map

// Object: Mapped<Hy, Covered, Moebius>
typedef struct HtHyMapped { Moebius map; HtHyCovered inner; } HtHyMapped;
inline __global const HtHyCovered *ht_hy_mapped__inner__gc(__global const HtHyMapped *s) { return &s->inner; }
#define $Self ObjectHtHyMapped
#define $self object_ht_hy_mapped
#define $Base HtHyMapped
#define $base ht_hy_mapped
#define $Geo Hy
#define $geo hy
#define $Map Moebius
#define $map mo
#define $Object HtHyCovered
#define $object ht_hy_covered
#define $Cache HtHyCoveredCache
#define $cache ht_hy_covered_cache
#include <object/mapped.inl>
#undef $Self
#undef $self
#undef $Base
#undef $base
#undef $Geo
#undef $geo
#undef $Map
#undef $map
#undef $Object
#undef $object
#undef $Cache
#undef $cache

// Object: Vec<Mapped<..>>
#define $Self HtHyVector
#define $self ht_hy_vector
#define $Element HtHyMapped
#define $element_size 128
#include <container/vector.inl>
#undef $Self
#undef $self
#undef $Element
#undef $element_size
typedef struct HtHyVectorCache { usize index; HtHyCoveredCache inner; } HtHyVectorCache;
typedef HtHyVector ObjectHtHyVector;
#define $Self ObjectHtHyVector
#define $self object_ht_hy_vector
#define $Base HtHyVector
#define $base ht_hy_vector
#define $Cache HtHyVectorCache
#define $cache ht_hy_vector_cache
#define $Geo Hy
#define $geo hy
#define $Object ObjectHtHyMapped
#define $object object_ht_hy_mapped
#define $ObjectCache HtHyCoveredCache
#define $object_cache ht_hy_covered_cache
#include <object/vector.inl>
#undef $Self
#undef $self
#undef $Base
#undef $base
#undef $Cache
#undef $cache
#undef $Geo
#undef $geo
#undef $Object
#undef $object
#undef $ObjectCache
#undef $object_cache

// Hop counter around the object detect the scene loop calls (harness instrumentation).
typedef HtHyVector CountedHy;
static real counted_hy_detect(__global const CountedHy *self, Context *context, HtHyVectorCache *cache, LightHy *light) {
    t_stats.hops += 1;
    t_stats.object_tests += self->size;
    real d = object_ht_hy_vector_detect(self, context, cache, light);
    if (d > (real)-0.5f) t_stats.hits += 1;
    return d;
}
static bool counted_hy_interact(__global const CountedHy *self, Context *context, HtHyVectorCache *cache, LightHy *light, color3 *emission) {
    return object_ht_hy_vector_interact(self, context, cache, light, emission);
}

// View: Mapped<Hy, PointView, Moebius>
typedef struct HtHyView { Moebius map; PointViewHy inner; } HtHyView;
#define $Self ViewHtHyView
#define $self view_ht_hy_view
#define $Base HtHyView
#define $base ht_hy_view
#define $Geo Hy
#define $geo hy
#define $Map Moebius
#define $map mo
#define $View PointViewHy
#define $view point_view_hy
#include <view/mapped.inl>
#undef $Self
#undef $self
#undef $Base
#undef $base
#undef $Geo
#undef $geo
#undef $Map
#undef $map
#undef $View
#undef $view

// Background: ConstBg
#define $Geo Hy
#define $geo hy
#include <background/constant.inl>
#undef $Geo
#undef $geo

// Scene
typedef struct HtHyScene { HtHyView view; ConstBg background; HtHyVector *object; } HtHyScene;
inline __global const ViewHtHyView *ht_hy_scene__view__gc(__global const HtHyScene *s) { return &s->view; }
inline __global const CountedHy *ht_hy_scene__object__gc(__global const HtHyScene *s) { return s->object; }
inline __global const ConstBg *ht_hy_scene__background__gc(__global const HtHyScene *s) { return &s->background; }
#define $Self HtHyScene
#define $self ht_hy_scene
#define $Geo Hy
#define $geo hy
#define $View ViewHtHyView
#define $view view_ht_hy_view
#define $Object CountedHy
#define $object counted_hy
#define $ObjectCache HtHyVectorCache
#define $object_cache ht_hy_vector_cache
#define $Background ConstBg
#define $background const_bg_hy
#define $light_hops g_light_hops
#include <render/scene.inl>
#undef $Self
#undef $self
#undef $Geo
#undef $geo
#undef $View
#undef $view
#undef $Object
#undef $object
#undef $ObjectCache
#undef $object_cache
#undef $Background
#undef $background
#undef $light_hops

// ============================================================================ euclidean
typedef struct HtEuChoice { usize index; } HtEuChoice;
inline __global const void *ht_eu_choice__Plane__gc(__global const HtEuChoice *) { return NULL; }
inline __global const Plane *ht_eu_choice__Plane__field_0__gc(__global const void *) { return NULL; }
inline __global const void *ht_eu_choice__Sphere__gc(__global const HtEuChoice *) { return NULL; }
inline __global const Sphere *ht_eu_choice__Sphere__field_0__gc(__global const void *) { return NULL; }
typedef HtEuChoice ShapeHtEuChoice;
#define $Self ShapeHtEuChoice
#define $self shape_ht_eu_choice
#define $Geo Eu
#define $geo eu
#define $shape_choice_detect_list \
    shape_choice_detect_variant(ht_eu_choice, 0, plane_eu, Plane) \
    shape_choice_detect_variant(ht_eu_choice, 1, sphere_eu, Sphere)
#include <shape/choice/impl.inl>
#undef $Self
#undef $self
#undef $Geo
#undef $geo
#undef $shape_choice_detect_list

typedef struct HtEuCovered { HtMixture material; HtEuChoice shape; } HtEuCovered;
typedef struct HtEuCoveredCache { EuDir normal; } HtEuCoveredCache;
inline __global const ShapeHtEuChoice *ht_eu_covered__shape__gc(__global const HtEuCovered *s) { return &s->shape; }
inline __global const HtMixture *ht_eu_covered__material__gc(__global const HtEuCovered *s) { return &s->material; }
#define $Self HtEuCovered
#define $self ht_eu_covered
#define $Geo Eu
#define $geo eu
#define $Shape ShapeHtEuChoice
#define $shape shape_ht_eu_choice
#define $Material HtMixture
#define $material ht_mixture
#define $Cache HtEuCoveredCache
#define $cache ht_eu_covered_cache
#include <object/covered.inl>
#undef $Self
#undef $self
#undef $Geo
#undef $geo
#undef $Shape
#undef $shape
#undef $Material
#undef $material
#undef $Cache
#undef $cache

#define $Geo Eu
#define $geo eu
#define $Map Homogenous3
#define $map hom3
#include <geometry/ray_map.inl>
#undef $Geo
#undef $geo
#undef $Map
#undef $map

typedef struct HtEuMapped { Homogenous3 map; HtEuCovered inner; } HtEuMapped;
inline __global const HtEuCovered *ht_eu_mapped__inner__gc(__global const HtEuMapped *s) { return &s->inner; }
#define $Self ObjectHtEuMapped
#define $self object_ht_eu_mapped
#define $Base HtEuMapped
#define $base ht_eu_mapped
#define $Geo Eu
#define $geo eu
#define $Map Homogenous3
#define $map hom3
#define $Object HtEuCovered
#define $object ht_eu_covered
#define $Cache HtEuCoveredCache
#define $cache ht_eu_covered_cache
#include <object/mapped.inl>
#undef $Self
#undef $self
#undef $Base
#undef $base
#undef $Geo
#undef $geo
#undef $Map
#undef $map
#undef $Object
#undef $object
#undef $Cache
#undef $cache

#define $Self HtEuVector
#define $self ht_eu_vector
#define $Element HtEuMapped
#define $element_size 128
#include <container/vector.inl>
#undef $Self
#undef $self
#undef $Element
#undef $element_size
typedef struct HtEuVectorCache { usize index; HtEuCoveredCache inner; } HtEuVectorCache;
typedef HtEuVector ObjectHtEuVector;
#define $Self ObjectHtEuVector
#define $self object_ht_eu_vector
#define $Base HtEuVector
#define $base ht_eu_vector
#define $Cache HtEuVectorCache
#define $cache ht_eu_vector_cache
#define $Geo Eu
#define $geo eu
#define $Object ObjectHtEuMapped
#define $object object_ht_eu_mapped
#define $ObjectCache HtEuCoveredCache
#define $object_cache ht_eu_covered_cache
#include <object/vector.inl>
#undef $Self
#undef $self
#undef $Base
#undef $base
#undef $Cache
#undef $cache
#undef $Geo
#undef $geo
#undef $Object
#undef $object
#undef $ObjectCache
#undef $object_cache

typedef HtEuVector CountedEu;
static real counted_eu_detect(__global const CountedEu *self, Context *context, HtEuVectorCache *cache, LightEu *light) {
    t_stats.hops += 1;
    t_stats.object_tests += self->size;
    real d = object_ht_eu_vector_detect(self, context, cache, light);
    if (d > (real)-0.5f) t_stats.hits += 1;
    return d;
}
static bool counted_eu_interact(__global const CountedEu *self, Context *context, HtEuVectorCache *cache, LightEu *light, color3 *emission) {
    return object_ht_eu_vector_interact(self, context, cache, light, emission);
}

typedef struct HtEuView { Homogenous3 map; PointViewEu inner; } HtEuView;
#define $Self ViewHtEuView
#define $self view_ht_eu_view
#define $Base HtEuView
#define $base ht_eu_view
#define $Geo Eu
#define $geo eu
#define $Map Homogenous3
#define $map hom3
#define $View PointViewEu
#define $view point_view_eu
#include <view/mapped.inl>
#undef $Self
#undef $self
#undef $Base
#undef $base
#undef $Geo
#undef $geo
#undef $Map
#undef $map
#undef $View
#undef $view

#define $Geo Eu
#define $geo eu
#include <background/constant.inl>
#undef $Geo
#undef $geo

typedef struct HtEuScene { HtEuView view; ConstBg background; HtEuVector *object; } HtEuScene;
inline __global const ViewHtEuView *ht_eu_scene__view__gc(__global const HtEuScene *s) { return &s->view; }
inline __global const CountedEu *ht_eu_scene__object__gc(__global const HtEuScene *s) { return s->object; }
inline __global const ConstBg *ht_eu_scene__background__gc(__global const HtEuScene *s) { return &s->background; }
#define $Self HtEuScene
#define $self ht_eu_scene
#define $Geo Eu
#define $geo eu
#define $View ViewHtEuView
#define $view view_ht_eu_view
#define $Object CountedEu
#define $object counted_eu
#define $ObjectCache HtEuVectorCache
#define $object_cache ht_eu_vector_cache
#define $Background ConstBg
#define $background const_bg_eu
#define $light_hops g_light_hops
#include <render/scene.inl>
#undef $Self
#undef $self
#undef $Geo
#undef $geo
#undef $View
#undef $view
#undef $Object
#undef $object
#undef $ObjectCache
#undef $object_cache
#undef $Background
#undef $background
#undef $light_hops

// ============================================================================ parsing
// Serialized layout (AddressWidth X32 or X64, double_support=false), little-endian.
// Offsets (derived in hypertrace_b200/scene.py) follow
// type-macros/src/entity.rs:7-186 (align = lcm of fields, fields aligned, size rounded
// to align) with float3 padded to 16 bytes (types/src/primitive/vector.rs:95-106).

static float rd_f(const uint8_t *b, size_t off) { float v; std::memcpy(&v, b + off, 4); return v; }
static uint32_t rd_u(const uint8_t *b, size_t off) { uint32_t v; std::memcpy(&v, b + off, 4); return v; }

enum { RECIPE_HY = 1, RECIPE_EU = 2 };
enum { OBJ_STRIDE = 128 };

static void parse_mixture(const uint8_t *o, HtMixture *m) {
    // Mixture starts 32 bytes into the object record (after the 32-byte map).
    m->diffuse.material.color = color3(rd_f(o, 32), rd_f(o, 36), rd_f(o, 40));
    m->diffuse.portion = (real)rd_f(o, 48);
    m->specular.portion = (real)rd_f(o, 64);
    m->luminous.material.emission = color3(rd_f(o, 80), rd_f(o, 84), rd_f(o, 88));
    m->luminous.portion = (real)rd_f(o, 96);
}

static Moebius parse_moebius(const uint8_t *b, size_t off) {
    Moebius m;
    m.v = comp2x2(
        (real)rd_f(b, off + 0), (real)rd_f(b, off + 4), (real)rd_f(b, off + 8), (real)rd_f(b, off + 12),
        (real)rd_f(b, off + 16), (real)rd_f(b, off + 20), (real)rd_f(b, off + 24), (real)rd_f(b, off + 28));
    return m;
}
static Homogenous3 parse_hom3(const uint8_t *b, size_t off) {
    Homogenous3 m;
    m.outer.v = real3((real)rd_f(b, off + 0), (real)rd_f(b, off + 4), (real)rd_f(b, off + 8));
    m.inner.v = quat((real)rd_f(b, off + 16), (real)rd_f(b, off + 20), (real)rd_f(b, off + 24), (real)rd_f(b, off + 28));
    return m;
}

struct ParsedScene {
    int recipe = 0;
    HtHyScene hy;
    HtEuScene eu;
    std::vector<uint8_t> storage;
};

static int parse_scene(int recipe, const uint8_t *b, size_t len, ParsedScene *ps) {
    ps->recipe = recipe;
    if (recipe == RECIPE_HY) {
        if (len < 128) return -1;
        ps->hy.view.map = parse_moebius(b, 0);
        ps->hy.view.inner.fov = (real)rd_f(b, 32);
        ps->hy.background.color = color3(rd_f(b, 64), rd_f(b, 68), rd_f(b, 72));
        uint32_t n = rd_u(b, 96);
        if (len < 128 + (size_t)n * OBJ_STRIDE) return -1;
        ps->storage.assign(sizeof(HtHyVector) + (n ? n : 1) * sizeof(HtHyMapped), 0);
        HtHyVector *v = reinterpret_cast<HtHyVector *>(ps->storage.data());
        v->size = n;
        for (uint32_t i = 0; i < n; ++i) {
            const uint8_t *o = b + 128 + (size_t)i * OBJ_STRIDE;
            HtHyMapped *e = &v->elements[i];
            e->map = parse_moebius(o, 0);
            parse_mixture(o, &e->inner.material);
            e->inner.shape.index = rd_u(o, 112);
        }
        ps->hy.object = v;
        return 0;
    } else if (recipe == RECIPE_EU) {
        if (len < 80) return -1;
        ps->eu.view.map = parse_hom3(b, 0);
        ps->eu.view.inner.fov = (real)rd_f(b, 32);
        ps->eu.background.color = color3(rd_f(b, 48), rd_f(b, 52), rd_f(b, 56));
        uint32_t n = rd_u(b, 64);
        if (len < 80 + (size_t)n * OBJ_STRIDE) return -1;
        ps->storage.assign(sizeof(HtEuVector) + (n ? n : 1) * sizeof(HtEuMapped), 0);
        HtEuVector *v = reinterpret_cast<HtEuVector *>(ps->storage.data());
        v->size = n;
        for (uint32_t i = 0; i < n; ++i) {
            const uint8_t *o = b + 80 + (size_t)i * OBJ_STRIDE;
            HtEuMapped *e = &v->elements[i];
            e->map = parse_hom3(o, 0);
            parse_mixture(o, &e->inner.material);
            e->inner.shape.index = rd_u(o, 112);
        }
        ps->eu.object = v;
        return 0;
    }
    return -2;
}

// ============================================================================ render
// Restatement of kernel/ocl/render/render.cl:6-27 for one pixel (host vector
// constructors in place of the OpenCL literals).
static void render_pixel(const ParsedScene &ps, uint32_t W, uint32_t H, uint32_t px,
                         float *canvas4, uint32_t *seed) {
    uint32_t x = px % W, y = px / W;
    real2 pos = real2(
        (real)(2 * x + 1) - (real)W,
        (real)H - (real)(2 * y + 1)
    ) / (real)H;
    real2 size = real2((real)2 / (real)H);

    Context context;
    context.rng.state = *seed;
    color3 c;
    if (ps.recipe == RECIPE_HY) {
        c = ht_hy_scene_sample(&ps.hy, &context, pos, size);
    } else {
        c = ht_eu_scene_sample(&ps.eu, &context, pos, size);
    }
    t_stats.samples += 1;
    canvas4[0] += c.x;
    canvas4[1] += c.y;
    canvas4[2] += c.z;
    canvas4[3] += 1.0f;
    *seed = context.rng.state;
}

static std::mutex g_mutex;

extern "C" {

// Renders `passes` passes over the listed pixels (pixel index = x + W*y of a W x H
// image), accumulating into canvas[4*i..] and advancing seeds[i] exactly as
// `passes` successive launches of the reference kernel would.
// threads <= 0 uses std::thread::hardware_concurrency().
// stats (optional) receives {samples, hops, object_tests, hits}.
int htref_render(int recipe, uint32_t hops, const uint8_t *scene, size_t scene_len,
                 uint32_t W, uint32_t H, const uint32_t *pixels, size_t n_pixels,
                 uint32_t passes, float *canvas, uint32_t *seeds, int threads,
                 uint64_t *stats) {
    std::lock_guard<std::mutex> lock(g_mutex);
    ParsedScene ps;
    int rc = parse_scene(recipe, scene, scene_len, &ps);
    if (rc != 0) return rc;
    if (hops == 0) return -3;
    g_light_hops = hops;
    if (threads <= 0) threads = (int)std::thread::hardware_concurrency();
    if (threads < 1) threads = 1;
    std::atomic<size_t> next{0};
    std::vector<RefStats> per(threads);
    const size_t CHUNK = 64;
    auto worker = [&](int tid) {
        t_stats = RefStats{0, 0, 0, 0};
        for (;;) {
            size_t start = next.fetch_add(CHUNK);
            if (start >= n_pixels) break;
            size_t end = start + CHUNK < n_pixels ? start + CHUNK : n_pixels;
            for (size_t i = start; i < end; ++i) {
                for (uint32_t p = 0; p < passes; ++p) {
                    render_pixel(ps, W, H, pixels[i], canvas + 4 * i, seeds + i);
                }
            }
        }
        per[tid] = t_stats;
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < threads; ++t) pool.emplace_back(worker, t);
    worker(0);
    for (auto &t : pool) t.join();
    if (stats) {
        RefStats s{0, 0, 0, 0};
        for (auto &p : per) {
            s.samples += p.samples; s.hops += p.hops;
            s.object_tests += p.object_tests; s.hits += p.hits;
        }
        stats[0] = s.samples; stats[1] = s.hops; stats[2] = s.object_tests; stats[3] = s.hits;
    }
    return 0;
}

// Precision of `real` this library was built with (4 or 8 bytes).
int htref_real_size(void) { return (int)sizeof(real); }

// The reference RNG stream (kernel/ocl/random.cc:8-14): n successive uniforms.
void htref_rng_uniforms(uint32_t seed, uint32_t n, double *out, uint32_t *state_out) {
    Rng rng = rng_init(seed);
    for (uint32_t i = 0; i < n; ++i) out[i] = (double)random_uniform(&rng);
    if (state_out) *state_out = rng.state;
}

// One cosine-weighted hemisphere draw (kernel/ocl/random.cc:53-59).
void htref_hemisphere_cosine(uint32_t seed, uint32_t n, double *out3, uint32_t *state_out) {
    Rng rng = rng_init(seed);
    for (uint32_t i = 0; i < n; ++i) {
        real3 v = random_hemisphere_cosine(&rng);
        out3[3 * i + 0] = v.x; out3[3 * i + 1] = v.y; out3[3 * i + 2] = v.z;
    }
    if (state_out) *state_out = rng.state;
}

// Moebius ray map of a hyperbolic ray (geometry/ray_map.inl:15-21 with mo_* maps).
void htref_ray_hy_map(const float *m8, const double *start4, const double *dir4, double *out8) {
    Moebius m;
    m.v = comp2x2((real)m8[0], (real)m8[1], (real)m8[2], (real)m8[3],
                  (real)m8[4], (real)m8[5], (real)m8[6], (real)m8[7]);
    RayHy r;
    r.start = quat((real)start4[0], (real)start4[1], (real)start4[2], (real)start4[3]);
    r.direction = quat((real)dir4[0], (real)dir4[1], (real)dir4[2], (real)dir4[3]);
    RayHy o = ray_hy_map_mo(r, m);
    for (int i = 0; i < 4; ++i) { out8[i] = o.start[i]; out8[4 + i] = o.direction[i]; }
}

}  // extern "C"
