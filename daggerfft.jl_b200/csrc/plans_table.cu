// Generated by gen_plans.py -- do not edit.
#include "static_plans.h"
namespace dfft {
extern const StaticPlan kPlans_f32_0[]; extern const int kPlansCount_f32_0;
extern const StaticPlan kPlans_f32_1[]; extern const int kPlansCount_f32_1;
extern const StaticPlan kPlans_f32_2[]; extern const int kPlansCount_f32_2;
extern const StaticPlan kPlans_f32_3[]; extern const int kPlansCount_f32_3;
extern const StaticPlan kPlans_f32_4[]; extern const int kPlansCount_f32_4;
extern const StaticPlan kPlans_f32_5[]; extern const int kPlansCount_f32_5;
extern const StaticPlan kPlans_f64_0[]; extern const int kPlansCount_f64_0;
extern const StaticPlan kPlans_f64_1[]; extern const int kPlansCount_f64_1;
extern const StaticPlan kPlans_f64_2[]; extern const int kPlansCount_f64_2;
extern const StaticPlan kPlans_f64_3[]; extern const int kPlansCount_f64_3;
extern const StaticPlan kPlans_f64_4[]; extern const int kPlansCount_f64_4;
extern const StaticPlan kPlans_f64_5[]; extern const int kPlansCount_f64_5;
const StaticPlanTable kTable_f32[] = {
  {kPlans_f32_0, &kPlansCount_f32_0},
  {kPlans_f32_1, &kPlansCount_f32_1},
  {kPlans_f32_2, &kPlansCount_f32_2},
  {kPlans_f32_3, &kPlansCount_f32_3},
  {kPlans_f32_4, &kPlansCount_f32_4},
  {kPlans_f32_5, &kPlansCount_f32_5},
};
const StaticPlanTable kTable_f64[] = {
  {kPlans_f64_0, &kPlansCount_f64_0},
  {kPlans_f64_1, &kPlansCount_f64_1},
  {kPlans_f64_2, &kPlansCount_f64_2},
  {kPlans_f64_3, &kPlansCount_f64_3},
  {kPlans_f64_4, &kPlansCount_f64_4},
  {kPlans_f64_5, &kPlansCount_f64_5},
};
const int kTableParts = 6;
}  // namespace dfft
