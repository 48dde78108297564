// Generated by gen_plans.py -- do not edit.
#include "static_plans.h"
namespace dfft {
template __global__ void axis_pass_static<double,true,1024,6,1,6>(const PassDesc);
template __global__ void axis_pass_static<double,false,1024,6,1,6>(const PassDesc);
template __global__ void axis_pass_static<double,true,512,16,1,16>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,16,1,16>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,16,1,16>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,16,1,16>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,30,5,6,5>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,30,5,6,5>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,30,5,6,5>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,30,5,6,5>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,50,5,10,5>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,50,5,10,5>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,50,5,10,5>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,50,5,10,5>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,80,8,10,8>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,80,8,10,8>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,80,8,10,8>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,80,8,10,8>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,120,10,12,10>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,120,10,12,10>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,120,10,12,10>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,120,10,12,10>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,160,10,10,16>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,160,10,10,16>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,160,10,10,16>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,160,10,10,16>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,225,15,15,15>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,225,15,15,15>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,225,15,15,15>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,225,15,15,15>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,288,36,6,6,8>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,288,36,6,6,8>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,288,36,6,6,8>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,288,36,6,6,8>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,384,48,6,8,8>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,384,48,6,8,8>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,384,48,6,8,8>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,384,48,6,8,8>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,1024,486,81,6,3,3,3,3>(const PassDesc);
template __global__ void axis_pass_static<double,false,1024,486,81,6,3,3,3,3>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,4,486,81,6,3,3,3,3>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,486,81,6,3,3,3,3>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,1024,625,125,5,5,5,5>(const PassDesc);
template __global__ void axis_pass_static<double,false,1024,625,125,5,5,5,5>(const PassDesc);
template __global__ void axis_pass_static<double,true,512,750,50,15,10,5>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,750,50,15,10,5>(const PassDesc);
template __global__ void axis_pass_static<double,true,512,960,80,12,10,8>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,960,80,12,10,8>(const PassDesc);
template __global__ void axis_pass_static<double,true,512,1152,96,12,12,8>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,1152,96,12,12,8>(const PassDesc);
template __global__ void axis_pass_static<double,true,512,1350,90,15,15,6>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,1350,90,15,15,6>(const PassDesc);
template __global__ void axis_pass_static<double,true,512,1620,108,15,12,3,3>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,1620,108,15,12,3,3>(const PassDesc);
template __global__ void axis_pass_static<double,true,512,2000,200,10,5,5,8>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,2000,200,10,5,5,8>(const PassDesc);
extern const StaticPlan kPlans_f64_5[];
extern const int kPlansCount_f64_5;
const StaticPlan kPlans_f64_5[] = {
  {6, 1, 1, {6}, 1024, (const void*)&axis_pass_static<double,true,1024,6,1,6>, (const void*)&axis_pass_static<double,false,1024,6,1,6>, nullptr, nullptr, 512, 0},
  {16, 1, 1, {16}, 512, (const void*)&axis_pass_static<double,true,512,16,1,16>, (const void*)&axis_pass_static<double,false,512,16,1,16>, (const void*)&axis_pass_pipe<double,512,false,8,16,1,16>, (const void*)&axis_pass_pipe<double,512,true,0,16,1,16>, 512, 8},
  {30, 5, 2, {6,5}, 512, (const void*)&axis_pass_static<double,true,512,30,5,6,5>, (const void*)&axis_pass_static<double,false,512,30,5,6,5>, (const void*)&axis_pass_pipe<double,512,false,8,30,5,6,5>, (const void*)&axis_pass_pipe<double,512,true,0,30,5,6,5>, 512, 8},
  {50, 5, 2, {10,5}, 512, (const void*)&axis_pass_static<double,true,512,50,5,10,5>, (const void*)&axis_pass_static<double,false,512,50,5,10,5>, (const void*)&axis_pass_pipe<double,512,false,8,50,5,10,5>, (const void*)&axis_pass_pipe<double,512,true,0,50,5,10,5>, 512, 8},
  {80, 8, 2, {10,8}, 512, (const void*)&axis_pass_static<double,true,512,80,8,10,8>, (const void*)&axis_pass_static<double,false,512,80,8,10,8>, (const void*)&axis_pass_pipe<double,512,false,8,80,8,10,8>, (const void*)&axis_pass_pipe<double,512,true,0,80,8,10,8>, 512, 8},
  {120, 10, 2, {12,10}, 512, (const void*)&axis_pass_static<double,true,512,120,10,12,10>, (const void*)&axis_pass_static<double,false,512,120,10,12,10>, (const void*)&axis_pass_pipe<double,512,false,8,120,10,12,10>, (const void*)&axis_pass_pipe<double,512,true,0,120,10,12,10>, 512, 8},
  {160, 10, 2, {10,16}, 512, (const void*)&axis_pass_static<double,true,512,160,10,10,16>, (const void*)&axis_pass_static<double,false,512,160,10,10,16>, (const void*)&axis_pass_pipe<double,512,false,8,160,10,10,16>, (const void*)&axis_pass_pipe<double,512,true,0,160,10,10,16>, 512, 8},
  {225, 15, 2, {15,15}, 512, (const void*)&axis_pass_static<double,true,512,225,15,15,15>, (const void*)&axis_pass_static<double,false,512,225,15,15,15>, (const void*)&axis_pass_pipe<double,512,false,8,225,15,15,15>, (const void*)&axis_pass_pipe<double,512,true,0,225,15,15,15>, 512, 8},
  {288, 36, 3, {6,6,8}, 512, (const void*)&axis_pass_static<double,true,512,288,36,6,6,8>, (const void*)&axis_pass_static<double,false,512,288,36,6,6,8>, (const void*)&axis_pass_pipe<double,512,false,8,288,36,6,6,8>, (const void*)&axis_pass_pipe<double,512,true,0,288,36,6,6,8>, 512, 8},
  {384, 48, 3, {6,8,8}, 512, (const void*)&axis_pass_static<double,true,512,384,48,6,8,8>, (const void*)&axis_pass_static<double,false,512,384,48,6,8,8>, (const void*)&axis_pass_pipe<double,512,false,8,384,48,6,8,8>, (const void*)&axis_pass_pipe<double,512,true,0,384,48,6,8,8>, 512, 8},
  {486, 81, 5, {6,3,3,3,3}, 1024, (const void*)&axis_pass_static<double,true,1024,486,81,6,3,3,3,3>, (const void*)&axis_pass_static<double,false,1024,486,81,6,3,3,3,3>, (const void*)&axis_pass_pipe<double,512,false,4,486,81,6,3,3,3,3>, (const void*)&axis_pass_pipe<double,512,true,0,486,81,6,3,3,3,3>, 512, 4},
  {625, 125, 4, {5,5,5,5}, 1024, (const void*)&axis_pass_static<double,true,1024,625,125,5,5,5,5>, (const void*)&axis_pass_static<double,false,1024,625,125,5,5,5,5>, nullptr, nullptr, 512, 0},
  {750, 50, 3, {15,10,5}, 512, (const void*)&axis_pass_static<double,true,512,750,50,15,10,5>, (const void*)&axis_pass_static<double,false,512,750,50,15,10,5>, nullptr, nullptr, 512, 0},
  {960, 80, 3, {12,10,8}, 512, (const void*)&axis_pass_static<double,true,512,960,80,12,10,8>, (const void*)&axis_pass_static<double,false,512,960,80,12,10,8>, nullptr, nullptr, 512, 0},
  {1152, 96, 3, {12,12,8}, 512, (const void*)&axis_pass_static<double,true,512,1152,96,12,12,8>, (const void*)&axis_pass_static<double,false,512,1152,96,12,12,8>, nullptr, nullptr, 512, 0},
  {1350, 90, 3, {15,15,6}, 512, (const void*)&axis_pass_static<double,true,512,1350,90,15,15,6>, (const void*)&axis_pass_static<double,false,512,1350,90,15,15,6>, nullptr, nullptr, 512, 0},
  {1620, 108, 4, {15,12,3,3}, 512, (const void*)&axis_pass_static<double,true,512,1620,108,15,12,3,3>, (const void*)&axis_pass_static<double,false,512,1620,108,15,12,3,3>, nullptr, nullptr, 512, 0},
  {2000, 200, 4, {10,5,5,8}, 512, (const void*)&axis_pass_static<double,true,512,2000,200,10,5,5,8>, (const void*)&axis_pass_static<double,false,512,2000,200,10,5,5,8>, nullptr, nullptr, 512, 0},
};
const int kPlansCount_f64_5 = 18;
}  // namespace dfft
