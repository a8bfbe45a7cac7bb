//! 512^3 R2C f32 forward + normalised inverse on a 4x8 virtual pencil grid,
//! the way a pencil-rs caller uses `R2cPlan` (distributed/r2c.rs:518-628):
//! build the plan, fill its input layout, transform, check the round trip.

use pencil_fft_b200::{DistributedLayout, MpiTopology, R2cPlan, Result};

fn main() -> Result<()> {
    let topology = MpiTopology::new([4, 8]);
    let plan = R2cPlan::<f32, 3, 2>::from_shape_with_selection_and_layout(
        &topology,
        [512, 512, 512],
        &[],
        None,
        DistributedLayout::default(),
    )?;
    // every virtual rank's local array, concatenated in rank order
    let n = plan.input_len();
    let host: Vec<f32> = (0..n).map(|i| ((i * 7919) % 2001) as f32 / 1000.0 - 1.0).collect();
    let input = pencil_fft_b200::DeviceBuffer::from_host(&host)?;
    let mut spectrum = plan.allocate_output()?;
    let mut back = plan.allocate_input()?;
    let mut ws = plan.allocate_workspace()?;
    let t_fwd = plan.forward_with_timing(&input, &mut spectrum, &mut ws)?;
    let t_inv = plan.inverse_with_timing(&spectrum, &mut back, &mut ws)?;
    let out = back.to_host()?;
    let (mut num, mut den) = (0f64, 0f64);
    for (a, b) in host.iter().zip(out.iter()) {
        num += ((a - b) as f64).powi(2);
        den += (*a as f64).powi(2);
    }
    println!(
        "forward passes {:?} ms, inverse {:?} ms, round-trip rel-L2 {:.2e}",
        t_fwd,
        t_inv,
        (num / den).sqrt()
    );
    Ok(())
}
