// oracle/_ref driver, second part: the scene types of the reference's `hy` and `eu` examples,
// instantiated from the reference's own kernel templates and compiled as host C++.
//
// TEST INFRASTRUCTURE ONLY (the checker). Nothing in the product links it.
//
//   recipe 3  SceneImpl<Hyperbolic3, Mapped<PointView, Moebius>,
//               Vec<Mapped<Choice{PlaneStar(TiledPlane<M, Pentastar, 2>),
//                 PlanePenta(TiledPlane<M, Pentagonal, 2>), HoroHexa(TiledHorosphere<M, Hexagonal, 3>),
//                 HoroSquare(TiledHorosphere<M, Square, 4>)}, Moebius>>, ConstBg, H>,
//             M = Emissive<Mixture{diffuse: Colored<Lambertian>, specular: Specular,
//                                  transparent: Transparent}>      (main/examples/hy.rs:35-75)
//   recipe 4  SceneImpl<Euclidean3, Mapped<PointView, Homogenous3>,
//               Vec<Mapped<Covered<Choice{Plane, Sphere, Cube}, Mixture{diffuse: Colored<Lambertian>,
//                 specular: Specular, refractive: Colored<Refractive>}>, Shift3>>, GradBg, H>
//                                                                  (main/examples/eu.rs:30-44)
//   recipe 5  a compound Euclidean type no example builds, for the containers and maps the
//             examples leave out: SceneImpl<Euclidean3, Mapped<PointView, Homogenous3>,
//               Mapped<Covered<Vec<Mapped<Choice{Plane, Sphere, Cube}, Chain<Shift3, Linear3>>>,
//                 Mixture{Colored<Lambertian>, Specular, Colored<Refractive>}>,
//                 Chain<Linear3, Shift3>>, GradBg, H>
// Generated struct text and getters follow type-macros/src/source.rs:14-92,171-178,190 and the
// object choice macros (objects/src/object/choice.rs, kernel/ocl/object/choice/macros.hh);
// the template instantiation pattern is that of kernel/ocl/render/test/scene_hy.cpp.
// Scene bytes (types/src/io.rs layout) are parsed into the host structs below; the byte
// offsets are the ones hypertrace_b200/types.py computes from the layout rules.

#include <cstdint>
#include <cstring>
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
#include <shape/eu/cube.hh>
#include <material/lambertian.hh>
#include <material/specular.hh>
#include <material/transparent.hh>
#include <material/refractive.hh>
#include <view/point/hy.hh>
#include <view/point/eu.hh>
#include <background/constant.hh>
#include <background/gradient.hh>
#include <transform/homogenous.hh>
#include <transform/shift.hh>
#include <transform/linear.hh>
#include <shape/choice/macros.hh>
#include <object/choice/macros.hh>
#include <material/mixture/macros.hh>

namespace {
uint g_ext_hops = 1;
struct ExtStats { uint64_t samples, hops, object_tests, hits; };
thread_local ExtStats t_ext;
}  // namespace

// ============================================================================ hy example
// Material M = Emissive<Mixture{Colored<Lambertian>, Specular, Transparent}>
typedef struct TlColoredLambertian { color3 color; } TlColoredLambertian;
inline __global const Lambertian *tl_colored_lambertian__inner__gc(__global const TlColoredLambertian *) { return NULL; }
#define $Self TlColoredLambertian
#define $self tl_colored_lambertian
#define $Material Lambertian
#define $material lambertian
#include <material/colored.inl>
#undef $Self
#undef $self
#undef $Material
#undef $material

typedef struct TlCompDiffuse { TlColoredLambertian material; real portion; } TlCompDiffuse;
inline __global const TlColoredLambertian *tl_comp_diffuse__material__gc(__global const TlCompDiffuse *s) { return &s->material; }
typedef struct TlCompSpecular { real portion; } TlCompSpecular;
inline __global const Specular *tl_comp_specular__material__gc(__global const TlCompSpecular *) { return NULL; }
typedef struct TlCompTransparent { real portion; } TlCompTransparent;
inline __global const Transparent *tl_comp_transparent__material__gc(__global const TlCompTransparent *) { return NULL; }
typedef struct TlMixture { TlCompDiffuse diffuse; TlCompSpecular specular; TlCompTransparent transparent; } TlMixture;
#define $Self TlMixture
#define $self tl_mixture
#define $mixture_interact_list \
    mixture_interact_component(tl_colored_lambertian, tl_comp_diffuse, diffuse) \
    mixture_interact_component(specular, tl_comp_specular, specular) \
    mixture_interact_component(transparent, tl_comp_transparent, transparent)
#include <material/mixture/impl.inl>
#undef $Self
#undef $self
#undef $mixture_interact_list

typedef struct TlMaterial { color3 emission; TlMixture inner; } TlMaterial;
inline __global const TlMixture *tl_material__inner__gc(__global const TlMaterial *s) { return &s->inner; }
#define $Self TlMaterial
#define $self tl_material
#define $Material TlMixture
#define $material tl_mixture
#include <material/emissive.inl>
#undef $Self
#undef $self
#undef $Material
#undef $material

// TiledPlane<M, K, 2> (struct generated by derive(EntitySource): materials as Array{elements})
typedef struct TlMatArray2 { TlMaterial elements[2]; } TlMatArray2;
typedef struct TlPlaneCache { HyDir normal; } TlPlaneCache;
typedef struct TlPlaneStar { TlMatArray2 materials; TlMaterial border_material; real cell_size; real border_width; } TlPlaneStar;
typedef struct TlPlanePenta { TlMatArray2 materials; TlMaterial border_material; real cell_size; real border_width; } TlPlanePenta;

#define $Self TlPlaneStar
#define $self tl_plane_star
#define $Cache TlPlaneCache
#define $cache tl_plane_cache
#define $Material TlMaterial
#define $material tl_material
#define $material_count 2
#define $tiling_type PLANE_HY_TILING_PENTASTAR
#include <object/hy/tiled_plane/impl.inl>
#undef $Self
#undef $self
#undef $tiling_type

#define $Self TlPlanePenta
#define $self tl_plane_penta
#define $tiling_type PLANE_HY_TILING_PENTAGONAL
#include <object/hy/tiled_plane/impl.inl>
#undef $Self
#undef $self
#undef $Cache
#undef $cache
#undef $Material
#undef $material
#undef $material_count
#undef $tiling_type

// TiledHorosphere<M, K, N> (struct defined by the template itself)
#define $Self TlHoroHexa
#define $self tl_horo_hexa
#define $Material TlMaterial
#define $material tl_material
#define $material_count 3
#define $tiling_type HOROSPHERE_TILING_HEXAGONAL
#include <object/hy/tiled_horosphere/impl.inl>
#undef $Self
#undef $self
#undef $material_count
#undef $tiling_type

#define $Self TlHoroSquare
#define $self tl_horo_square
#define $material_count 4
#define $tiling_type HOROSPHERE_TILING_SQUARE
#include <object/hy/tiled_horosphere/impl.inl>
#undef $Self
#undef $self
#undef $Material
#undef $material
#undef $material_count
#undef $tiling_type

// Choice { PlaneStar, PlanePenta, HoroHexa, HoroSquare } (object_choice!, hy.rs:66-73)
typedef struct TlChoice {
    usize index;
    TlPlaneStar PlaneStar;
    TlPlanePenta PlanePenta;
    TlHoroHexa HoroHexa;
    TlHoroSquare HoroSquare;
} TlChoice;
inline __global const void *tl_choice__PlaneStar__gc(__global const TlChoice *s) { return &s->PlaneStar; }
inline __global const TlPlaneStar *tl_choice__PlaneStar__field_0__gc(__global const void *p) { return (const TlPlaneStar *)p; }
inline __global const void *tl_choice__PlanePenta__gc(__global const TlChoice *s) { return &s->PlanePenta; }
inline __global const TlPlanePenta *tl_choice__PlanePenta__field_0__gc(__global const void *p) { return (const TlPlanePenta *)p; }
inline __global const void *tl_choice__HoroHexa__gc(__global const TlChoice *s) { return &s->HoroHexa; }
inline __global const TlHoroHexa *tl_choice__HoroHexa__field_0__gc(__global const void *p) { return (const TlHoroHexa *)p; }
inline __global const void *tl_choice__HoroSquare__gc(__global const TlChoice *s) { return &s->HoroSquare; }
inline __global const TlHoroSquare *tl_choice__HoroSquare__field_0__gc(__global const void *p) { return (const TlHoroSquare *)p; }
typedef struct TlChoiceCache {
    TlPlaneCache PlaneStar;
    TlPlaneCache PlanePenta;
    TiledHorosphereCache HoroHexa;
    TiledHorosphereCache HoroSquare;
} TlChoiceCache;
inline TlPlaneCache *tl_choice_cache__PlaneStar(TlChoiceCache *c) { return &c->PlaneStar; }
inline TlPlaneCache *tl_choice_cache__PlanePenta(TlChoiceCache *c) { return &c->PlanePenta; }
inline TiledHorosphereCache *tl_choice_cache__HoroHexa(TlChoiceCache *c) { return &c->HoroHexa; }
inline TiledHorosphereCache *tl_choice_cache__HoroSquare(TlChoiceCache *c) { return &c->HoroSquare; }
typedef TlChoice ObjectTlChoice;
#define $Self ObjectTlChoice
#define $self object_tl_choice
#define $Geo Hy
#define $geo hy
#define $Cache TlChoiceCache
#define $cache tl_choice_cache
#define $object_choice_detect_list \
    object_choice_detect_variant(tl_choice, 0, tl_plane_star, PlaneStar) \
    object_choice_detect_variant(tl_choice, 1, tl_plane_penta, PlanePenta) \
    object_choice_detect_variant(tl_choice, 2, tl_horo_hexa, HoroHexa) \
    object_choice_detect_variant(tl_choice, 3, tl_horo_square, HoroSquare)
#define $object_choice_interact_list \
    object_choice_interact_variant(tl_choice, 0, tl_plane_star, PlaneStar) \
    object_choice_interact_variant(tl_choice, 1, tl_plane_penta, PlanePenta) \
    object_choice_interact_variant(tl_choice, 2, tl_horo_hexa, HoroHexa) \
    object_choice_interact_variant(tl_choice, 3, tl_horo_square, HoroSquare)
#include <object/choice/impl.inl>
#undef $Self
#undef $self
#undef $Geo
#undef $geo
#undef $Cache
#undef $cache
#undef $object_choice_detect_list
#undef $object_choice_interact_list

#define $Geo Hy
#define $geo hy
#define $Map Moebius
#define $map mo
#include <geometry/ray_map.inl>
#undef $Geo
#undef $geo
#undef $Map
#undef $map

typedef struct TlMapped { Moebius map; TlChoice inner; } TlMapped;
inline __global const TlChoice *tl_mapped__inner__gc(__global const TlMapped *s) { return &s->inner; }
#define $Self ObjectTlMapped
#define $self object_tl_mapped
#define $Base TlMapped
#define $base tl_mapped
#define $Geo Hy
#define $geo hy
#define $Map Moebius
#define $map mo
#define $Object ObjectTlChoice
#define $object object_tl_choice
#define $Cache TlChoiceCache
#define $cache tl_choice_cache
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

#define $Self TlVector
#define $self tl_vector
#define $Element TlMapped
#define $element_size 384
#include <container/vector.inl>
#undef $Self
#undef $self
#undef $Element
#undef $element_size
typedef struct TlVectorCache { usize index; TlChoiceCache inner; } TlVectorCache;
typedef TlVector ObjectTlVector;
#define $Self ObjectTlVector
#define $self object_tl_vector
#define $Base TlVector
#define $base tl_vector
#define $Cache TlVectorCache
#define $cache tl_vector_cache
#define $Geo Hy
#define $geo hy
#define $Object ObjectTlMapped
#define $object object_tl_mapped
#define $ObjectCache TlChoiceCache
#define $object_cache tl_choice_cache
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

typedef TlVector CountedTl;
static real counted_tl_detect(__global const CountedTl *self, Context *context, TlVectorCache *cache, LightHy *light) {
    t_ext.hops += 1;
    t_ext.object_tests += self->size;
    real d = object_tl_vector_detect(self, context, cache, light);
    if (d > (real)-0.5f) t_ext.hits += 1;
    return d;
}
static bool counted_tl_interact(__global const CountedTl *self, Context *context, TlVectorCache *cache, LightHy *light, color3 *emission) {
    return object_tl_vector_interact(self, context, cache, light, emission);
}

typedef struct TlView { Moebius map; PointViewHy inner; } TlView;
#define $Self ViewTlView
#define $self view_tl_view
#define $Base TlView
#define $base tl_view
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

#define $Geo Hy
#define $geo hy
#include <background/constant.inl>
#undef $Geo
#undef $geo

typedef struct TlScene { TlView view; ConstBg background; TlVector *object; } TlScene;
inline __global const ViewTlView *tl_scene__view__gc(__global const TlScene *s) { return &s->view; }
inline __global const CountedTl *tl_scene__object__gc(__global const TlScene *s) { return s->object; }
inline __global const ConstBg *tl_scene__background__gc(__global const TlScene *s) { return &s->background; }
#define $Self TlScene
#define $self tl_scene
#define $Geo Hy
#define $geo hy
#define $View ViewTlView
#define $view view_tl_view
#define $Object CountedTl
#define $object counted_tl
#define $ObjectCache TlVectorCache
#define $object_cache tl_vector_cache
#define $Background ConstBg
#define $background const_bg_hy
#define $light_hops g_ext_hops
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

// ============================================================================ eu example
typedef struct GrChoice { usize index; } GrChoice;
inline __global const void *gr_choice__Plane__gc(__global const GrChoice *) { return NULL; }
inline __global const PlaneEu *gr_choice__Plane__field_0__gc(__global const void *) { return NULL; }
inline __global const void *gr_choice__Sphere__gc(__global const GrChoice *) { return NULL; }
inline __global const SphereEu *gr_choice__Sphere__field_0__gc(__global const void *) { return NULL; }
inline __global const void *gr_choice__Cube__gc(__global const GrChoice *) { return NULL; }
inline __global const CubeEu *gr_choice__Cube__field_0__gc(__global const void *) { return NULL; }
typedef GrChoice ShapeGrChoice;
#define $Self ShapeGrChoice
#define $self shape_gr_choice
#define $Geo Eu
#define $geo eu
#define $shape_choice_detect_list \
    shape_choice_detect_variant(gr_choice, 0, plane_eu, Plane) \
    shape_choice_detect_variant(gr_choice, 1, sphere_eu, Sphere) \
    shape_choice_detect_variant(gr_choice, 2, cube_eu, Cube)
#include <shape/choice/impl.inl>
#undef $Self
#undef $self
#undef $Geo
#undef $geo
#undef $shape_choice_detect_list

typedef struct GrColoredLambertian { color3 color; } GrColoredLambertian;
inline __global const Lambertian *gr_colored_lambertian__inner__gc(__global const GrColoredLambertian *) { return NULL; }
#define $Self GrColoredLambertian
#define $self gr_colored_lambertian
#define $Material Lambertian
#define $material lambertian
#include <material/colored.inl>
#undef $Self
#undef $self
#undef $Material
#undef $material
typedef struct GrColoredRefractive { color3 color; Refractive inner; } GrColoredRefractive;
inline __global const Refractive *gr_colored_refractive__inner__gc(__global const GrColoredRefractive *s) { return &s->inner; }
#define $Self GrColoredRefractive
#define $self gr_colored_refractive
#define $Material Refractive
#define $material refractive
#include <material/colored.inl>
#undef $Self
#undef $self
#undef $Material
#undef $material

typedef struct GrCompDiffuse { GrColoredLambertian material; real portion; } GrCompDiffuse;
inline __global const GrColoredLambertian *gr_comp_diffuse__material__gc(__global const GrCompDiffuse *s) { return &s->material; }
typedef struct GrCompSpecular { real portion; } GrCompSpecular;
inline __global const Specular *gr_comp_specular__material__gc(__global const GrCompSpecular *) { return NULL; }
typedef struct GrCompRefractive { GrColoredRefractive material; real portion; } GrCompRefractive;
inline __global const GrColoredRefractive *gr_comp_refractive__material__gc(__global const GrCompRefractive *s) { return &s->material; }
typedef struct GrMixture { GrCompDiffuse diffuse; GrCompSpecular specular; GrCompRefractive refractive; } GrMixture;
#define $Self GrMixture
#define $self gr_mixture
#define $mixture_interact_list \
    mixture_interact_component(gr_colored_lambertian, gr_comp_diffuse, diffuse) \
    mixture_interact_component(specular, gr_comp_specular, specular) \
    mixture_interact_component(gr_colored_refractive, gr_comp_refractive, refractive)
#include <material/mixture/impl.inl>
#undef $Self
#undef $self
#undef $mixture_interact_list

typedef struct GrCovered { GrMixture material; GrChoice shape; } GrCovered;
typedef struct GrCoveredCache { EuDir normal; } GrCoveredCache;
inline __global const ShapeGrChoice *gr_covered__shape__gc(__global const GrCovered *s) { return &s->shape; }
inline __global const GrMixture *gr_covered__material__gc(__global const GrCovered *s) { return &s->material; }
#define $Self GrCovered
#define $self gr_covered
#define $Geo Eu
#define $geo eu
#define $Shape ShapeGrChoice
#define $shape shape_gr_choice
#define $Material GrMixture
#define $material gr_mixture
#define $Cache GrCoveredCache
#define $cache gr_covered_cache
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
#define $Map Shift3
#define $map shf3
#include <geometry/ray_map.inl>
#undef $Geo
#undef $geo
#undef $Map
#undef $map

typedef struct GrMapped { Shift3 map; GrCovered inner; } GrMapped;
inline __global const GrCovered *gr_mapped__inner__gc(__global const GrMapped *s) { return &s->inner; }
#define $Self ObjectGrMapped
#define $self object_gr_mapped
#define $Base GrMapped
#define $base gr_mapped
#define $Geo Eu
#define $geo eu
#define $Map Shift3
#define $map shf3
#define $Object GrCovered
#define $object gr_covered
#define $Cache GrCoveredCache
#define $cache gr_covered_cache
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

#define $Self GrVector
#define $self gr_vector
#define $Element GrMapped
#define $element_size 128
#include <container/vector.inl>
#undef $Self
#undef $self
#undef $Element
#undef $element_size
typedef struct GrVectorCache { usize index; GrCoveredCache inner; } GrVectorCache;
typedef GrVector ObjectGrVector;
#define $Self ObjectGrVector
#define $self object_gr_vector
#define $Base GrVector
#define $base gr_vector
#define $Cache GrVectorCache
#define $cache gr_vector_cache
#define $Geo Eu
#define $geo eu
#define $Object ObjectGrMapped
#define $object object_gr_mapped
#define $ObjectCache GrCoveredCache
#define $object_cache gr_covered_cache
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

typedef GrVector CountedGr;
static real counted_gr_detect(__global const CountedGr *self, Context *context, GrVectorCache *cache, LightEu *light) {
    t_ext.hops += 1;
    t_ext.object_tests += self->size;
    real d = object_gr_vector_detect(self, context, cache, light);
    if (d > (real)-0.5f) t_ext.hits += 1;
    return d;
}
static bool counted_gr_interact(__global const CountedGr *self, Context *context, GrVectorCache *cache, LightEu *light, color3 *emission) {
    return object_gr_vector_interact(self, context, cache, light, emission);
}

#define $Geo Eu
#define $geo eu
#define $Map Homogenous3
#define $map hom3
#include <geometry/ray_map.inl>
#undef $Geo
#undef $geo
#undef $Map
#undef $map

typedef struct GrView { Homogenous3 map; PointViewEu inner; } GrView;
#define $Self ViewGrView
#define $self view_gr_view
#define $Base GrView
#define $base gr_view
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

typedef struct GrScene { GrView view; GradBg background; GrVector *object; } GrScene;
inline __global const ViewGrView *gr_scene__view__gc(__global const GrScene *s) { return &s->view; }
inline __global const CountedGr *gr_scene__object__gc(__global const GrScene *s) { return s->object; }
inline __global const GradBg *gr_scene__background__gc(__global const GrScene *s) { return &s->background; }
#define $Self GrScene
#define $self gr_scene
#define $Geo Eu
#define $geo eu
#define $View ViewGrView
#define $view view_gr_view
#define $Object CountedGr
#define $object counted_gr
#define $ObjectCache GrVectorCache
#define $object_cache gr_vector_cache
#define $Background GradBg
#define $background grad_bg
#define $light_hops g_ext_hops
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

// ============================================================================ compound type
// Chain<Shift3, Linear3> and Chain<Linear3, Shift3> (transform/chain.inl)
#define $Self CpChainSL
#define $self cp_chain_sl
#define $Outer Shift3
#define $outer shf3
#define $Inner Linear3
#define $inner lin3
#define $elem real3
#include <transform/chain.inl>
#undef $Self
#undef $self
#undef $Outer
#undef $outer
#undef $Inner
#undef $inner
#undef $elem
#define $Self CpChainLS
#define $self cp_chain_ls
#define $Outer Linear3
#define $outer lin3
#define $Inner Shift3
#define $inner shf3
#define $elem real3
#include <transform/chain.inl>
#undef $Self
#undef $self
#undef $Outer
#undef $outer
#undef $Inner
#undef $inner
#undef $elem

#define $Geo Eu
#define $geo eu
#define $Map CpChainSL
#define $map cp_chain_sl
#include <geometry/ray_map.inl>
#undef $Map
#undef $map
#define $Map CpChainLS
#define $map cp_chain_ls
#include <geometry/ray_map.inl>
#undef $Map
#undef $map
#undef $Geo
#undef $geo

// Mapped<Choice{Plane, Sphere, Cube}, Chain<Shift3, Linear3>> as a shape (shape/mapped.inl)
typedef struct CpMShape { CpChainSL map; GrChoice inner; } CpMShape;
inline __global const ShapeGrChoice *cp_mshape__inner__gc(__global const CpMShape *s) { return &s->inner; }
#define $Self ShapeCpMShape
#define $self shape_cp_mshape
#define $Base CpMShape
#define $base cp_mshape
#define $Geo Eu
#define $geo eu
#define $Map CpChainSL
#define $map cp_chain_sl
#define $Shape ShapeGrChoice
#define $shape shape_gr_choice
#include <shape/mapped.inl>
#undef $Self
#undef $self
#undef $Base
#undef $base
#undef $Geo
#undef $geo
#undef $Map
#undef $map
#undef $Shape
#undef $shape

// Vec<..> as a shape (shape/vector.inl)
#define $Self CpShapeVector
#define $self cp_shape_vector
#define $Element CpMShape
#define $element_size 192
#include <container/vector.inl>
#undef $Self
#undef $self
#undef $Element
#undef $element_size
#define $Self ShapeCpVector
#define $self shape_cp_vector
#define $Base CpShapeVector
#define $base cp_shape_vector
#define $Geo Eu
#define $geo eu
#define $Shape ShapeCpMShape
#define $shape shape_cp_mshape
#include <shape/vector.inl>
#undef $Self
#undef $self
#undef $Base
#undef $base
#undef $Geo
#undef $geo
#undef $Shape
#undef $shape

typedef struct CpCovered { GrMixture material; CpShapeVector *shape; } CpCovered;
typedef struct CpCoveredCache { EuDir normal; } CpCoveredCache;
inline __global const ShapeCpVector *cp_covered__shape__gc(__global const CpCovered *s) { return s->shape; }
inline __global const GrMixture *cp_covered__material__gc(__global const CpCovered *s) { return &s->material; }
#define $Self CpCovered
#define $self cp_covered
#define $Geo Eu
#define $geo eu
#define $Shape ShapeCpVector
#define $shape shape_cp_vector
#define $Material GrMixture
#define $material gr_mixture
#define $Cache CpCoveredCache
#define $cache cp_covered_cache
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

typedef struct CpMapped { CpChainLS map; CpCovered inner; } CpMapped;
inline __global const CpCovered *cp_mapped__inner__gc(__global const CpMapped *s) { return &s->inner; }
#define $Self ObjectCpMapped
#define $self object_cp_mapped
#define $Base CpMapped
#define $base cp_mapped
#define $Geo Eu
#define $geo eu
#define $Map CpChainLS
#define $map cp_chain_ls
#define $Object CpCovered
#define $object cp_covered
#define $Cache CpCoveredCache
#define $cache cp_covered_cache
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

typedef CpMapped CountedCp;
static real counted_cp_detect(__global const CountedCp *self, Context *context, CpCoveredCache *cache, LightEu *light) {
    t_ext.hops += 1;
    t_ext.object_tests += 1;
    real d = object_cp_mapped_detect(self, context, cache, light);
    if (d > (real)-0.5f) t_ext.hits += 1;
    return d;
}
static bool counted_cp_interact(__global const CountedCp *self, Context *context, CpCoveredCache *cache, LightEu *light, color3 *emission) {
    return object_cp_mapped_interact(self, context, cache, light, emission);
}

typedef struct CpScene { GrView view; GradBg background; CpMapped object; } CpScene;
inline __global const ViewGrView *cp_scene__view__gc(__global const CpScene *s) { return &s->view; }
inline __global const CountedCp *cp_scene__object__gc(__global const CpScene *s) { return &s->object; }
inline __global const GradBg *cp_scene__background__gc(__global const CpScene *s) { return &s->background; }
#define $Self CpScene
#define $self cp_scene
#define $Geo Eu
#define $geo eu
#define $View ViewGrView
#define $view view_gr_view
#define $Object CountedCp
#define $object counted_cp
#define $ObjectCache CpCoveredCache
#define $object_cache cp_covered_cache
#define $Background GradBg
#define $background grad_bg
#define $light_hops g_ext_hops
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
namespace {

float rdf(const uint8_t *b, size_t off) { float v; std::memcpy(&v, b + off, 4); return v; }
uint32_t rdu(const uint8_t *b, size_t off) { uint32_t v; std::memcpy(&v, b + off, 4); return v; }
color3 rdc(const uint8_t *b, size_t off) { return color3(rdf(b, off), rdf(b, off + 4), rdf(b, off + 8)); }
real3 rdr3(const uint8_t *b, size_t off) { return real3((real)rdf(b, off), (real)rdf(b, off + 4), (real)rdf(b, off + 8)); }
Moebius rdmo(const uint8_t *b, size_t off) {
    Moebius m;
    m.v = comp2x2((real)rdf(b, off + 0), (real)rdf(b, off + 4), (real)rdf(b, off + 8), (real)rdf(b, off + 12),
                  (real)rdf(b, off + 16), (real)rdf(b, off + 20), (real)rdf(b, off + 24), (real)rdf(b, off + 28));
    return m;
}

// Material M (64 bytes): emission @0, diffuse color @16, diffuse portion @32,
// specular portion @48, transparent portion @52.
TlMaterial rd_tl_material(const uint8_t *b, size_t off) {
    TlMaterial m;
    m.emission = rdc(b, off);
    m.inner.diffuse.material.color = rdc(b, off + 16);
    m.inner.diffuse.portion = (real)rdf(b, off + 32);
    m.inner.specular.portion = (real)rdf(b, off + 48);
    m.inner.transparent.portion = (real)rdf(b, off + 52);
    return m;
}
template <typename T, int N> void rd_tiled(const uint8_t *b, size_t off, T *t, TlMaterial *mats, TlMaterial *border,
                                           real *cell, real *width) {
    for (int i = 0; i < N; ++i) mats[i] = rd_tl_material(b, off + 64 * i);
    *border = rd_tl_material(b, off + 64 * N);
    *cell = (real)rdf(b, off + 64 * N + 64);
    *width = (real)rdf(b, off + 64 * N + 68);
    (void)t;
}

constexpr size_t TL_STRIDE = 384, GR_STRIDE = 128, CP_STRIDE = 192;

// Linear3: 16 floats, rows padded (types/src/primitive/matrix.rs:117-165)
Linear3 rdlin(const uint8_t *b, size_t off) {
    Linear3 m;
    for (int i = 0; i < 16; ++i) m.v.s[i] = (real)rdf(b, off + 4 * i);
    return m;
}

struct ExtScene {
    int recipe = 0;
    TlScene tl;
    GrScene gr;
    CpScene cp;
    std::vector<uint8_t> storage;
};

int parse_ext(int recipe, const uint8_t *b, size_t len, ExtScene *s) {
    s->recipe = recipe;
    if (recipe == 3) {
        if (len < 128) return -1;
        s->tl.view.map = rdmo(b, 0);
        s->tl.view.inner.fov = (real)rdf(b, 32);
        s->tl.background.color = rdc(b, 64);
        const uint32_t n = rdu(b, 96);
        if (len < 128 + (size_t)n * TL_STRIDE) return -1;
        s->storage.assign(sizeof(TlVector) + (n ? n : 1) * sizeof(TlMapped), 0);
        TlVector *v = reinterpret_cast<TlVector *>(s->storage.data());
        v->size = n;
        for (uint32_t i = 0; i < n; ++i) {
            const uint8_t *o = b + 128 + (size_t)i * TL_STRIDE;
            TlMapped *e = &v->elements[i];
            e->map = rdmo(o, 0);
            const uint32_t k = rdu(o, 32);
            e->inner.index = k;
            const size_t p = 48;   // payload (usize index padded to the enum's alignment 16)
            if (k == 0) rd_tiled<TlPlaneStar, 2>(o, p, &e->inner.PlaneStar, e->inner.PlaneStar.materials.elements,
                                                 &e->inner.PlaneStar.border_material, &e->inner.PlaneStar.cell_size,
                                                 &e->inner.PlaneStar.border_width);
            else if (k == 1) rd_tiled<TlPlanePenta, 2>(o, p, &e->inner.PlanePenta, e->inner.PlanePenta.materials.elements,
                                                       &e->inner.PlanePenta.border_material, &e->inner.PlanePenta.cell_size,
                                                       &e->inner.PlanePenta.border_width);
            else if (k == 2) rd_tiled<TlHoroHexa, 3>(o, p, &e->inner.HoroHexa, e->inner.HoroHexa.materials,
                                                     &e->inner.HoroHexa.border_material, &e->inner.HoroHexa.cell_size,
                                                     &e->inner.HoroHexa.border_width);
            else if (k == 3) rd_tiled<TlHoroSquare, 4>(o, p, &e->inner.HoroSquare, e->inner.HoroSquare.materials,
                                                       &e->inner.HoroSquare.border_material, &e->inner.HoroSquare.cell_size,
                                                       &e->inner.HoroSquare.border_width);
            else return -1;
        }
        s->tl.object = v;
        return 0;
    }
    if (recipe == 4) {
        if (len < 128) return -1;
        s->gr.view.map.outer.v = rdr3(b, 0);
        s->gr.view.map.inner.v = quat((real)rdf(b, 16), (real)rdf(b, 20), (real)rdf(b, 24), (real)rdf(b, 28));
        s->gr.view.inner.fov = (real)rdf(b, 32);
        s->gr.background.direction = rdr3(b, 48);
        s->gr.background.colors[0] = rdc(b, 64);
        s->gr.background.colors[1] = rdc(b, 80);
        s->gr.background.power = rdf(b, 96);
        const uint32_t n = rdu(b, 112);
        if (len < 128 + (size_t)n * GR_STRIDE) return -1;
        s->storage.assign(sizeof(GrVector) + (n ? n : 1) * sizeof(GrMapped), 0);
        GrVector *v = reinterpret_cast<GrVector *>(s->storage.data());
        v->size = n;
        for (uint32_t i = 0; i < n; ++i) {
            const uint8_t *o = b + 128 + (size_t)i * GR_STRIDE;
            GrMapped *e = &v->elements[i];
            e->map.v = rdr3(o, 0);
            e->inner.material.diffuse.material.color = rdc(o, 16);
            e->inner.material.diffuse.portion = (real)rdf(o, 32);
            e->inner.material.specular.portion = (real)rdf(o, 48);
            e->inner.material.refractive.material.color = rdc(o, 64);
            e->inner.material.refractive.material.inner.index = (real)rdf(o, 80);
            e->inner.material.refractive.portion = (real)rdf(o, 96);
            e->inner.shape.index = rdu(o, 112);
            if (e->inner.shape.index > 2) return -1;
        }
        s->gr.object = v;
        return 0;
    }
    if (recipe == 5) {
        // view Homogenous3 @0, fov @32, GradBg @48..112, object @128: map Chain<Linear3, Shift3>
        // (linear @128, shift @192), material @256 (as recipe 4 at +240), shape Vec: count @384,
        // elements @448 + 192 i: map Chain<Shift3, Linear3> (shift @0, linear @64), choice @128.
        if (len < 448) return -1;
        s->cp.view.map.outer.v = rdr3(b, 0);
        s->cp.view.map.inner.v = quat((real)rdf(b, 16), (real)rdf(b, 20), (real)rdf(b, 24), (real)rdf(b, 28));
        s->cp.view.inner.fov = (real)rdf(b, 32);
        s->cp.background.direction = rdr3(b, 48);
        s->cp.background.colors[0] = rdc(b, 64);
        s->cp.background.colors[1] = rdc(b, 80);
        s->cp.background.power = rdf(b, 96);
        s->cp.object.map.outer = rdlin(b, 128);
        s->cp.object.map.inner.v = rdr3(b, 192);
        GrMixture &m = s->cp.object.inner.material;
        m.diffuse.material.color = rdc(b, 256);
        m.diffuse.portion = (real)rdf(b, 272);
        m.specular.portion = (real)rdf(b, 288);
        m.refractive.material.color = rdc(b, 304);
        m.refractive.material.inner.index = (real)rdf(b, 320);
        m.refractive.portion = (real)rdf(b, 336);
        const uint32_t n = rdu(b, 384);
        if (len < 448 + (size_t)n * CP_STRIDE) return -1;
        s->storage.assign(sizeof(CpShapeVector) + (n ? n : 1) * sizeof(CpMShape), 0);
        CpShapeVector *v = reinterpret_cast<CpShapeVector *>(s->storage.data());
        v->size = n;
        for (uint32_t i = 0; i < n; ++i) {
            const uint8_t *o = b + 448 + (size_t)i * CP_STRIDE;
            CpMShape *e = &v->elements[i];
            e->map.outer.v = rdr3(o, 0);
            e->map.inner = rdlin(o, 64);
            e->inner.index = rdu(o, 128);
            if (e->inner.index > 2) return -1;
        }
        s->cp.object.inner.shape = v;
        return 0;
    }
    return -2;
}

void render_ext_pixel(const ExtScene &s, uint32_t W, uint32_t H, uint32_t px, float *canvas4, uint32_t *seed) {
    uint32_t x = px % W, y = px / W;
    real2 pos = real2((real)(2 * x + 1) - (real)W, (real)H - (real)(2 * y + 1)) / (real)H;
    real2 size = real2((real)2 / (real)H);
    Context context;
    context.rng.state = *seed;
    color3 c = s.recipe == 3 ? tl_scene_sample(&s.tl, &context, pos, size)
             : s.recipe == 4 ? gr_scene_sample(&s.gr, &context, pos, size)
                             : cp_scene_sample(&s.cp, &context, pos, size);
    t_ext.samples += 1;
    canvas4[0] += c.x;
    canvas4[1] += c.y;
    canvas4[2] += c.z;
    canvas4[3] += 1.0f;
    *seed = context.rng.state;
}

std::mutex g_ext_mutex;

}  // namespace

extern "C" {

// htref_render for recipes 3, 4 and 5 (same arguments and semantics).
int htref_render_ext(int recipe, uint32_t hops, const uint8_t *scene, size_t scene_len, uint32_t W, uint32_t H,
                     const uint32_t *pixels, size_t n_pixels, uint32_t passes, float *canvas, uint32_t *seeds,
                     int threads, uint64_t *stats) {
    std::lock_guard<std::mutex> lock(g_ext_mutex);
    ExtScene s;
    int rc = parse_ext(recipe, scene, scene_len, &s);
    if (rc != 0) return rc;
    if (hops == 0) return -3;
    g_ext_hops = hops;
    if (threads <= 0) threads = (int)std::thread::hardware_concurrency();
    if (threads < 1) threads = 1;
    std::atomic<size_t> next{0};
    std::vector<ExtStats> per(threads);
    auto worker = [&](int tid) {
        t_ext = ExtStats{0, 0, 0, 0};
        for (;;) {
            size_t start = next.fetch_add(64);
            if (start >= n_pixels) break;
            size_t end = start + 64 < n_pixels ? start + 64 : n_pixels;
            for (size_t i = start; i < end; ++i)
                for (uint32_t p = 0; p < passes; ++p) render_ext_pixel(s, W, H, pixels[i], canvas + 4 * i, seeds + i);
        }
        per[tid] = t_ext;
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < threads; ++t) pool.emplace_back(worker, t);
    worker(0);
    for (auto &t : pool) t.join();
    if (stats) {
        ExtStats a{0, 0, 0, 0};
        for (auto &p : per) { a.samples += p.samples; a.hops += p.hops; a.object_tests += p.object_tests; a.hits += p.hits; }
        stats[0] = a.samples; stats[1] = a.hops; stats[2] = a.object_tests; stats[3] = a.hits;
    }
    return 0;
}

}  // extern "C"
