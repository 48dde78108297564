// Generated by gen_plans.py -- do not edit.
#include "static_plans.h"
namespace dfft {
template __global__ void axis_pass_static<float,true,1024,6,1,6>(const PassDesc);
template __global__ void axis_pass_static<float,false,1024,6,1,6>(const PassDesc);
template __global__ void axis_pass_static<float,true,1024,16,1,16>(const PassDesc);
template __global__ void axis_pass_static<float,false,1024,16,1,16>(const PassDesc);
template __global__ void axis_pass_pipe<float,1024,false,16,16,1,16>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<float,1024,true,0,16,1,16>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<float,true,1024,30,5,6,5>(const PassDesc);
template __global__ void axis_pass_static<float,false,1024,30,5,6,5>(const PassDesc);
template __global__ void axis_pass_pipe<float,1024,false,16,30,5,6,5>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<float,1024,true,0,30,5,6,5>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<float,true,1024,50,5,10,5>(const PassDesc);
template __global__ void axis_pass_static<float,false,1024,50,5,10,5>(const PassDesc);
template __global__ void axis_pass_pipe<float,1024,false,16,50,5,10,5>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<float,1024,true,0,50,5,10,5>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<float,true,1024,80,8,10,8>(const PassDesc);
template __global__ void axis_pass_static<float,false,1024,80,8,10,8>(const PassDesc);
template __global__ void axis_pass_pipe<float,1024,false,16,80,8,10,8>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<float,1024,true,0,80,8,10,8>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<float,true,512,120,10,12,10>(const PassDesc);
template __global__ void axis_pass_static<float,false,512,120,10,12,10>(const PassDesc);
template __global__ void axis_pass_pipe<float,512,false,16,120,10,12,10>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<float,512,true,0,120,10,12,10>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<float,true,512,160,10,10,16>(const PassDesc);
template __global__ void axis_pass_static<float,false,512,160,10,10,16>(const PassDesc);
template __global__ void axis_pass_pipe<float,512,false,16,160,10,10,16>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<float,512,true,0,160,10,10,16>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<float,true,1024,225,15,15,15>(const PassDesc);
template __global__ void axis_pass_static<float,false,1024,225,15,15,15>(const PassDesc);
template __global__ void axis_pass_pipe<float,1024,false,16,225,15,15,15>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<float,1024,true,0,225,15,15,15>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<float,true,1024,288,36,6,6,8>(const PassDesc);
template __global__ void axis_pass_static<float,false,1024,288,36,6,6,8>(const PassDesc);
template __global__ void axis_pass_pipe<float,1024,false,16,288,36,6,6,8>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<float,1024,true,0,288,36,6,6,8>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<float,true,1024,384,48,6,8,8>(const PassDesc);
template __global__ void axis_pass_static<float,false,1024,384,48,6,8,8>(const PassDesc);
template __global__ void axis_pass_pipe<float,1024,false,16,384,48,6,8,8>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<float,1024,true,0,384,48,6,8,8>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<float,true,1024,486,81,6,3,3,3,3>(const PassDesc);
template __global__ void axis_pass_static<float,false,1024,486,81,6,3,3,3,3>(const PassDesc);
template __global__ void axis_pass_pipe<float,1024,false,8,486,81,6,3,3,3,3>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<float,1024,true,0,486,81,6,3,3,3,3>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<float,true,1024,625,125,5,5,5,5>(const PassDesc);
template __global__ void axis_pass_static<float,false,1024,625,125,5,5,5,5>(const PassDesc);
template __global__ void axis_pass_pipe<float,1024,false,8,625,125,5,5,5,5>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<float,1024,true,0,625,125,5,5,5,5>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<float,true,512,750,50,15,10,5>(const PassDesc);
template __global__ void axis_pass_static<float,false,512,750,50,15,10,5>(const PassDesc);
template __global__ void axis_pass_pipe<float,512,false,8,750,50,15,10,5>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<float,512,true,0,750,50,15,10,5>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<float,true,512,960,80,12,10,8>(const PassDesc);
template __global__ void axis_pass_static<float,false,512,960,80,12,10,8>(const PassDesc);
template __global__ void axis_pass_pipe<float,512,false,4,960,80,12,10,8>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<float,512,true,0,960,80,12,10,8>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<float,true,1024,1152,96,12,12,8>(const PassDesc);
template __global__ void axis_pass_static<float,false,1024,1152,96,12,12,8>(const PassDesc);
template __global__ void axis_pass_static<float,true,512,1350,90,15,15,6>(const PassDesc);
template __global__ void axis_pass_static<float,false,512,1350,90,15,15,6>(const PassDesc);
template __global__ void axis_pass_static<float,true,512,1620,108,15,12,3,3>(const PassDesc);
template __global__ void axis_pass_static<float,false,512,1620,108,15,12,3,3>(const PassDesc);
template __global__ void axis_pass_static<float,true,1024,2000,200,10,5,5,8>(const PassDesc);
template __global__ void axis_pass_static<float,false,1024,2000,200,10,5,5,8>(const PassDesc);
template __global__ void axis_pass_static<float,true,512,2304,144,12,12,16>(const PassDesc);
template __global__ void axis_pass_static<float,false,512,2304,144,12,12,16>(const PassDesc);
template __global__ void axis_pass_static<float,true,512,2700,180,15,15,12>(const PassDesc);
template __global__ void axis_pass_static<float,false,512,2700,180,15,15,12>(const PassDesc);
template __global__ void axis_pass_static<float,true,1024,3200,320,10,5,8,8>(const PassDesc);
template __global__ void axis_pass_static<float,false,1024,3200,320,10,5,8,8>(const PassDesc);
template __global__ void axis_pass_static<float,true,512,3750,250,15,10,5,5>(const PassDesc);
template __global__ void axis_pass_static<float,false,512,3750,250,15,10,5,5>(const PassDesc);
extern const StaticPlan kPlans_f32_5[];
extern const int kPlansCount_f32_5;
const StaticPlan kPlans_f32_5[] = {
  {6, 1, 1, {6}, 1024, (const void*)&axis_pass_static<float,true,1024,6,1,6>, (const void*)&axis_pass_static<float,false,1024,6,1,6>, nullptr, nullptr, 1024, 0},
  {16, 1, 1, {16}, 1024, (const void*)&axis_pass_static<float,true,1024,16,1,16>, (const void*)&axis_pass_static<float,false,1024,16,1,16>, (const void*)&axis_pass_pipe<float,1024,false,16,16,1,16>, (const void*)&axis_pass_pipe<float,1024,true,0,16,1,16>, 1024, 16},
  {30, 5, 2, {6,5}, 1024, (const void*)&axis_pass_static<float,true,1024,30,5,6,5>, (const void*)&axis_pass_static<float,false,1024,30,5,6,5>, (const void*)&axis_pass_pipe<float,1024,false,16,30,5,6,5>, (const void*)&axis_pass_pipe<float,1024,true,0,30,5,6,5>, 1024, 16},
  {50, 5, 2, {10,5}, 1024, (const void*)&axis_pass_static<float,true,1024,50,5,10,5>, (const void*)&axis_pass_static<float,false,1024,50,5,10,5>, (const void*)&axis_pass_pipe<float,1024,false,16,50,5,10,5>, (const void*)&axis_pass_pipe<float,1024,true,0,50,5,10,5>, 1024, 16},
  {80, 8, 2, {10,8}, 1024, (const void*)&axis_pass_static<float,true,1024,80,8,10,8>, (const void*)&axis_pass_static<float,false,1024,80,8,10,8>, (const void*)&axis_pass_pipe<float,1024,false,16,80,8,10,8>, (const void*)&axis_pass_pipe<float,1024,true,0,80,8,10,8>, 1024, 16},
  {120, 10, 2, {12,10}, 512, (const void*)&axis_pass_static<float,true,512,120,10,12,10>, (const void*)&axis_pass_static<float,false,512,120,10,12,10>, (const void*)&axis_pass_pipe<float,512,false,16,120,10,12,10>, (const void*)&axis_pass_pipe<float,512,true,0,120,10,12,10>, 512, 16},
  {160, 10, 2, {10,16}, 512, (const void*)&axis_pass_static<float,true,512,160,10,10,16>, (const void*)&axis_pass_static<float,false,512,160,10,10,16>, (const void*)&axis_pass_pipe<float,512,false,16,160,10,10,16>, (const void*)&axis_pass_pipe<float,512,true,0,160,10,10,16>, 512, 16},
  {225, 15, 2, {15,15}, 1024, (const void*)&axis_pass_static<float,true,1024,225,15,15,15>, (const void*)&axis_pass_static<float,false,1024,225,15,15,15>, (const void*)&axis_pass_pipe<float,1024,false,16,225,15,15,15>, (const void*)&axis_pass_pipe<float,1024,true,0,225,15,15,15>, 1024, 16},
  {288, 36, 3, {6,6,8}, 1024, (const void*)&axis_pass_static<float,true,1024,288,36,6,6,8>, (const void*)&axis_pass_static<float,false,1024,288,36,6,6,8>, (const void*)&axis_pass_pipe<float,1024,false,16,288,36,6,6,8>, (const void*)&axis_pass_pipe<float,1024,true,0,288,36,6,6,8>, 1024, 16},
  {384, 48, 3, {6,8,8}, 1024, (const void*)&axis_pass_static<float,true,1024,384,48,6,8,8>, (const void*)&axis_pass_static<float,false,1024,384,48,6,8,8>, (const void*)&axis_pass_pipe<float,1024,false,16,384,48,6,8,8>, (const void*)&axis_pass_pipe<float,1024,true,0,384,48,6,8,8>, 1024, 16},
  {486, 81, 5, {6,3,3,3,3}, 1024, (const void*)&axis_pass_static<float,true,1024,486,81,6,3,3,3,3>, (const void*)&axis_pass_static<float,false,1024,486,81,6,3,3,3,3>, (const void*)&axis_pass_pipe<float,1024,false,8,486,81,6,3,3,3,3>, (const void*)&axis_pass_pipe<float,1024,true,0,486,81,6,3,3,3,3>, 1024, 8},
  {625, 125, 4, {5,5,5,5}, 1024, (const void*)&axis_pass_static<float,true,1024,625,125,5,5,5,5>, (const void*)&axis_pass_static<float,false,1024,625,125,5,5,5,5>, (const void*)&axis_pass_pipe<float,1024,false,8,625,125,5,5,5,5>, (const void*)&axis_pass_pipe<float,1024,true,0,625,125,5,5,5,5>, 1024, 8},
  {750, 50, 3, {15,10,5}, 512, (const void*)&axis_pass_static<float,true,512,750,50,15,10,5>, (const void*)&axis_pass_static<float,false,512,750,50,15,10,5>, (const void*)&axis_pass_pipe<float,512,false,8,750,50,15,10,5>, (const void*)&axis_pass_pipe<float,512,true,0,750,50,15,10,5>, 512, 8},
  {960, 80, 3, {12,10,8}, 512, (const void*)&axis_pass_static<float,true,512,960,80,12,10,8>, (const void*)&axis_pass_static<float,false,512,960,80,12,10,8>, (const void*)&axis_pass_pipe<float,512,false,4,960,80,12,10,8>, (const void*)&axis_pass_pipe<float,512,true,0,960,80,12,10,8>, 512, 4},
  {1152, 96, 3, {12,12,8}, 1024, (const void*)&axis_pass_static<float,true,1024,1152,96,12,12,8>, (const void*)&axis_pass_static<float,false,1024,1152,96,12,12,8>, nullptr, nullptr, 1024, 0},
  {1350, 90, 3, {15,15,6}, 512, (const void*)&axis_pass_static<float,true,512,1350,90,15,15,6>, (const void*)&axis_pass_static<float,false,512,1350,90,15,15,6>, nullptr, nullptr, 512, 0},
  {1620, 108, 4, {15,12,3,3}, 512, (const void*)&axis_pass_static<float,true,512,1620,108,15,12,3,3>, (const void*)&axis_pass_static<float,false,512,1620,108,15,12,3,3>, nullptr, nullptr, 512, 0},
  {2000, 200, 4, {10,5,5,8}, 1024, (const void*)&axis_pass_static<float,true,1024,2000,200,10,5,5,8>, (const void*)&axis_pass_static<float,false,1024,2000,200,10,5,5,8>, nullptr, nullptr, 1024, 0},
  {2304, 144, 3, {12,12,16}, 512, (const void*)&axis_pass_static<float,true,512,2304,144,12,12,16>, (const void*)&axis_pass_static<float,false,512,2304,144,12,12,16>, nullptr, nullptr, 512, 0},
  {2700, 180, 3, {15,15,12}, 512, (const void*)&axis_pass_static<float,true,512,2700,180,15,15,12>, (const void*)&axis_pass_static<float,false,512,2700,180,15,15,12>, nullptr, nullptr, 512, 0},
  {3200, 320, 4, {10,5,8,8}, 1024, (const void*)&axis_pass_static<float,true,1024,3200,320,10,5,8,8>, (const void*)&axis_pass_static<float,false,1024,3200,320,10,5,8,8>, nullptr, nullptr, 1024, 0},
  {3750, 250, 4, {15,10,5,5}, 512, (const void*)&axis_pass_static<float,true,512,3750,250,15,10,5,5>, (const void*)&axis_pass_static<float,false,512,3750,250,15,10,5,5>, nullptr, nullptr, 512, 0},
};
const int kPlansCount_f32_5 = 22;
}  // namespace dfft
